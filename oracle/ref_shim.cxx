// TEST INFRASTRUCTURE ONLY -- part of the oracle, never part of the product.
//
// C shim over the reference's own CPU build of the Green-function action
// (real-space/AngstromCube compiled with -DHAS_NO_CUDA, which turns every
// __global__ kernel into serial CPU loops, include/green_cuda.hxx:19-47).
// It builds plans programmatically (no Hmt.xml), fills the potential and the
// atom matrices directly (the MPI exchanges are switched off) and exposes
// the reference's action_t::multiply (include/green_action.hxx:140-176) and
// plan arrays to the parity tests through plain C functions.
//
// Only tests/, the smoke check and bench.py's CPU-baseline leg load the
// resulting library (oracle/_ref/libref_green.so).

#include <cstdint>
#include <cstring>
#include <cstdio>
#include <vector>
#include <complex>

#include "green_function.hxx"   // construct_Green_function, update_energy_parameter, update_phases
#include "green_action.hxx"     // green_action::action_t
#include "kinetic_plan.hxx"     // kinetic_plan::set_phase
#include "control.hxx"          // control::set
#include "sho_tools.hxx"        // sho_tools::nSHO
#include "sho_projection.hxx"   // sho_projection::get_sho_prefactors
#include "energy_contour.hxx"   // energy_contour::get_energy_mesh and its quadratures
#include "green_solver.hxx"     // green_solver_t (link stubs below)

// defined in src/energy_contour.cxx without a declaration in its header
namespace energy_contour {
std::vector<std::complex<double>> get_energy_mesh(std::vector<std::complex<double>> &w8, double kBT, double eBot,
                                                  unsigned nBot, unsigned nPar, unsigned nFer, int nPol, int echo);
}

namespace {

struct RefPlan {
    action_plan_t p;
    uint32_t n_blocks[3] = {0, 0, 0};
    std::vector<uint16_t> colIndex;     // copy of p.colindx, the action's colIndex argument
    double (*veff_cells)[64] = nullptr; // potential storage [max(nRows, ncells)][64]
    green_action::action_t<double,2,1,64> *act64 = nullptr;
    green_action::action_t<float ,2,1,64> *act32 = nullptr;
    ~RefPlan() { delete act64; delete act32; }
};

} // namespace

extern "C" {

// Geometry description, mirrored by tests/oracle python code.
struct ref_geometry_t {
    int32_t ng[3];          // grid points per direction (multiples of 4)
    int32_t bc[3];          // 0:isolated 1:periodic 2:vacuum 3:repeat
    double  hg[3];          // grid spacings
    double  r_trunc;        // green_function.truncation.radius
    double  sources[3];     // green_function.sources.x/.y/.z (-1: all)
    int32_t nFD;            // green_kinetic.range (4 or 8)
    double  proj_radius;    // green_function.projection.radius (in sigma)
    int32_t natoms;
    const double *xyzZinso; // [natoms*8]
    int32_t echo;
};

void* ref_plan_build(const ref_geometry_t *g) {
    char buf[64];
    control::set("green_function.potential.exchange", "0", -1);
    control::set("green_function.matrices.exchange", "0", -1);
    std::snprintf(buf, 64, "%.17g", g->r_trunc);  control::set("green_function.truncation.radius", buf, -1);
    std::snprintf(buf, 64, "%.17g", g->sources[0]); control::set("green_function.sources.x", buf, -1);
    std::snprintf(buf, 64, "%.17g", g->sources[1]); control::set("green_function.sources.y", buf, -1);
    std::snprintf(buf, 64, "%.17g", g->sources[2]); control::set("green_function.sources.z", buf, -1);
    std::snprintf(buf, 64, "%d", g->nFD);          control::set("green_kinetic.range", buf, -1);
    // control::get stores the default of a missing key on first use; the per-direction ranges
    // default to the (possibly reduced) global range, so clear them as a fresh process would
    control::set("green_kinetic.range.x", "", -1);
    control::set("green_kinetic.range.y", "", -1);
    control::set("green_kinetic.range.z", "", -1);
    std::snprintf(buf, 64, "%.17g", g->proj_radius); control::set("green_function.projection.radius", buf, -1);

    auto *rp = new RefPlan();
    uint32_t ng[3];
    int8_t bc[3];
    for (int d = 0; d < 3; ++d) { ng[d] = g->ng[d]; bc[d] = int8_t(g->bc[d]); rp->n_blocks[d] = ng[d] >> 2; }
    std::vector<double> xyzZinso(g->xyzZinso, g->xyzZinso + 8*size_t(g->natoms));
    auto const stat = green_function::construct_Green_function(rp->p, ng, bc, g->hg, xyzZinso, g->echo, 1);
    if (stat) { delete rp; return nullptr; }
    rp->colIndex = rp->p.colindx;
    // the reference reads Vloc[veff_index[inzb]] with veff_index = cube index inside the cell
    // (src/green_function.cxx:913-916, include/green_potential.hxx:90-91), so provide
    // storage for every cell cube (and at least nRows as the reference allocates)
    size_t const ncells = size_t(rp->n_blocks[0])*rp->n_blocks[1]*rp->n_blocks[2];
    size_t const nV = std::max(ncells, size_t(rp->p.nRows));
    free_memory(rp->p.Veff[0]);
    rp->veff_cells = get_memory<double[64]>(nV, 0, "Veff[0] (cells)");
    std::memset(rp->veff_cells, 0, nV*64*sizeof(double));
    rp->p.Veff[0] = rp->veff_cells;
    rp->p.echo = 0;
    return rp;
}

void ref_plan_free(void *h) {
    auto *rp = (RefPlan*)h;
    delete rp;
}

// sizes: [0]nnzb [1]nRows [2]nCols [3]nAtoms [4]nAtomImages [5]ncoeff_images
//        [6]ncoeffs [7..9]nlists[dd] [10..12]lists_nnz[dd] [13]SHOadd_nnz
//        [14]SHOprj_nnz(total) [15]SHOsum_nnz [16..18]FD_range[dd] [19]ncells
void ref_plan_sizes(void *h, int64_t *s) {
    auto &p = ((RefPlan*)h)->p;
    auto const &dp = p.dyadic_plan;
    s[0] = p.colindx.size(); s[1] = p.nRows; s[2] = p.nCols;
    s[3] = dp.nAtoms; s[4] = dp.nAtomImages;
    s[5] = dp.AtomImageStarts ? dp.AtomImageStarts[dp.nAtomImages] : 0;
    s[6] = dp.AtomStarts ? dp.AtomStarts[dp.nAtoms] : 0;
    for (int dd = 0; dd < 3; ++dd) {
        s[7 + dd] = p.kinetic[dd].sparse_.nRows();
        s[10 + dd] = p.kinetic[dd].sparse_.nNonzeros();
        s[16 + dd] = p.kinetic[dd].FD_range_;
    }
    s[13] = dp.sparse_SHOadd.nNonzeros();
    int64_t nprj{0};
    for (int irhs = 0; irhs < dp.nrhs; ++irhs) nprj += dp.sparse_SHOprj[irhs].nNonzeros();
    s[14] = nprj;
    s[15] = dp.sparse_SHOsum.nNonzeros();
    auto const *rp = (RefPlan*)h;
    s[19] = int64_t(rp->n_blocks[0])*rp->n_blocks[1]*rp->n_blocks[2];
}

// Export of the plan arrays (any pointer may be null to skip it).
struct ref_plan_export_t {
    uint32_t *rowstart;        // [nRows+1]
    uint16_t *colindx;         // [nnzb]
    uint32_t *rowindx;         // [nnzb]
    int32_t  *veff_index;      // [nnzb]
    uint32_t *subset;          // [nCols]
    float    *rowCubePos;      // [nRows][4]
    float    *colCubePos;      // [nCols][4]
    int16_t  *target_minus_source; // [nnzb][4]
    double   *grid_spacing_trunc;  // [3]
    double   *kinetic_prefactor;   // [3]
    uint32_t *lists_start[3];  // [nlists+1]
    int32_t  *lists[3];        // [lists_nnz]
    // dyadic plan
    uint32_t *AtomStarts;      // [nAtoms+1]
    int8_t   *AtomLmax;        // [nAtoms]
    double   *AtomSigma;       // [nAtoms]
    int64_t  *global_atom_ids; // [nAtoms]
    uint32_t *AtomImageIndex;  // [nAI]
    uint32_t *AtomImageStarts; // [nAI+1]
    double   *AtomImagePos;    // [nAI][4]
    int8_t   *AtomImageLmax;   // [nAI]
    int8_t   *AtomImageShift;  // [nAI][4]
    double   *AtomImagePhase;  // [nAI][4]
    double   *grid_spacing_dyadic; // [4]
    uint32_t *SHOadd_start;    // [nnzb+1]
    uint32_t *SHOadd_col;      // [SHOadd_nnz]
    uint32_t *SHOprj_start;    // [nCols][nAI+1] concatenated
    uint32_t *SHOprj_col;      // [SHOprj_nnz] concatenated over rhs
    uint32_t *SHOsum_start;    // [nAtoms+1]
    uint32_t *SHOsum_col;      // [SHOsum_nnz]
    double   *AtomMatrices;    // [nAtoms][2*nc*nc] concatenated (device-layout copy)
    double   *phase;           // [3][2][2]
};

void ref_plan_export(void *h, ref_plan_export_t const *e) {
    auto &p = ((RefPlan*)h)->p;
    auto const &dp = p.dyadic_plan;
    size_t const nnzb = p.colindx.size();
    if (e->rowstart) std::memcpy(e->rowstart, p.RowStart, (p.nRows + 1)*sizeof(uint32_t));
    if (e->colindx) std::memcpy(e->colindx, p.colindx.data(), nnzb*sizeof(uint16_t));
    if (e->rowindx) std::memcpy(e->rowindx, p.rowindx, nnzb*sizeof(uint32_t));
    if (e->veff_index) std::memcpy(e->veff_index, p.veff_index, nnzb*sizeof(int32_t));
    if (e->subset) std::memcpy(e->subset, p.subset.data(), p.nCols*sizeof(uint32_t));
    if (e->rowCubePos) std::memcpy(e->rowCubePos, p.rowCubePos, p.nRows*4*sizeof(float));
    if (e->colCubePos) std::memcpy(e->colCubePos, p.colCubePos, p.nCols*4*sizeof(float));
    if (e->target_minus_source) std::memcpy(e->target_minus_source, p.target_minus_source, nnzb*4*sizeof(int16_t));
    if (e->grid_spacing_trunc) std::memcpy(e->grid_spacing_trunc, p.grid_spacing_trunc, 3*sizeof(double));
    for (int dd = 0; dd < 3; ++dd) {
        auto const &k = p.kinetic[dd];
        if (e->kinetic_prefactor) e->kinetic_prefactor[dd] = k.prefactor_;
        if (e->lists_start[dd]) std::memcpy(e->lists_start[dd], k.sparse_.rowStart(), (k.sparse_.nRows() + 1)*sizeof(uint32_t));
        if (e->lists[dd]) std::memcpy(e->lists[dd], k.sparse_.colIndex(), k.sparse_.nNonzeros()*sizeof(int32_t));
    }
    uint32_t const nA = dp.nAtoms, nAI = dp.nAtomImages;
    if (e->AtomStarts && dp.AtomStarts) std::memcpy(e->AtomStarts, dp.AtomStarts, (nA + 1)*sizeof(uint32_t));
    if (e->AtomLmax && nA) std::memcpy(e->AtomLmax, dp.AtomLmax, nA);
    if (e->AtomSigma && nA) std::memcpy(e->AtomSigma, dp.AtomSigma, nA*sizeof(double));
    if (e->global_atom_ids) for (uint32_t i = 0; i < nA; ++i) e->global_atom_ids[i] = dp.global_atom_ids[i];
    if (e->AtomImageIndex && nAI) std::memcpy(e->AtomImageIndex, dp.AtomImageIndex, nAI*sizeof(uint32_t));
    if (e->AtomImageStarts && dp.AtomImageStarts) std::memcpy(e->AtomImageStarts, dp.AtomImageStarts, (nAI + 1)*sizeof(uint32_t));
    if (e->AtomImagePos && nAI) std::memcpy(e->AtomImagePos, dp.AtomImagePos, nAI*4*sizeof(double));
    if (e->AtomImageLmax && nAI) std::memcpy(e->AtomImageLmax, dp.AtomImageLmax, nAI);
    if (e->AtomImageShift && nAI) std::memcpy(e->AtomImageShift, dp.AtomImageShift, nAI*4);
    if (e->AtomImagePhase && nAI) std::memcpy(e->AtomImagePhase, dp.AtomImagePhase, nAI*4*sizeof(double));
    if (e->grid_spacing_dyadic) std::memcpy(e->grid_spacing_dyadic, dp.grid_spacing, 4*sizeof(double));
    if (e->SHOadd_start && dp.sparse_SHOadd.rowStart()) std::memcpy(e->SHOadd_start, dp.sparse_SHOadd.rowStart(), (dp.sparse_SHOadd.nRows() + 1)*sizeof(uint32_t));
    if (e->SHOadd_col && dp.sparse_SHOadd.colIndex()) std::memcpy(e->SHOadd_col, dp.sparse_SHOadd.colIndex(), dp.sparse_SHOadd.nNonzeros()*sizeof(uint32_t));
    if (e->SHOprj_start || e->SHOprj_col) {
        size_t off_s{0}, off_c{0};
        for (int irhs = 0; irhs < dp.nrhs; ++irhs) {
            auto const &sp = dp.sparse_SHOprj[irhs];
            if (e->SHOprj_start) {
                if (sp.rowStart()) std::memcpy(e->SHOprj_start + off_s, sp.rowStart(), (nAI + 1)*sizeof(uint32_t));
                else std::memset(e->SHOprj_start + off_s, 0, (nAI + 1)*sizeof(uint32_t));
            }
            off_s += nAI + 1;
            if (e->SHOprj_col && sp.nNonzeros()) std::memcpy(e->SHOprj_col + off_c, sp.colIndex(), sp.nNonzeros()*sizeof(uint32_t));
            off_c += sp.nNonzeros();
        }
    }
    if (e->SHOsum_start && dp.sparse_SHOsum.rowStart()) std::memcpy(e->SHOsum_start, dp.sparse_SHOsum.rowStart(), (dp.sparse_SHOsum.nRows() + 1)*sizeof(uint32_t));
    if (e->SHOsum_col && dp.sparse_SHOsum.colIndex()) std::memcpy(e->SHOsum_col, dp.sparse_SHOsum.colIndex(), dp.sparse_SHOsum.nNonzeros()*sizeof(uint32_t));
    if (e->AtomMatrices) {
        size_t off{0};
        for (uint32_t ia = 0; ia < nA; ++ia) {
            int const nc = sho_tools::nSHO(dp.AtomLmax[ia]);
            std::memcpy(e->AtomMatrices + off, dp.AtomMatrices[ia], 2*nc*nc*sizeof(double));
            off += 2*nc*nc;
        }
    }
    if (e->phase) std::memcpy(e->phase, p.phase, 12*sizeof(double));
}

// Potential given per cell cube: Vcell[ncells][64], cube index (iz*nby + iy)*nbx + ix,
// point index i64 = (i4z*4 + i4y)*4 + i4x (src/green_function.cxx:147-158).
void ref_set_potential(void *h, const double *Vcell) {
    auto *rp = (RefPlan*)h;
    size_t const ncells = size_t(rp->n_blocks[0])*rp->n_blocks[1]*rp->n_blocks[2];
    std::memcpy(rp->veff_cells, Vcell, ncells*64*sizeof(double));
}

// Atom matrices per original atom (already rescaled for unnormalized Hermite functions,
// src/energy_contour.cxx:307-323): concatenated [natoms][2][nc][nc] (hmt, ovl).
// They are placed where green_parallel::exchange would put them (src/green_function.cxx:192-208).
void ref_set_atom_matrices(void *h, const double *mats, const int64_t *offsets) {
    auto &dp = ((RefPlan*)h)->p.dyadic_plan;
    for (uint32_t iac = 0; iac < dp.nAtoms; ++iac) {
        auto const gid = dp.global_atom_ids[iac];
        int const nc = sho_tools::nSHO(dp.AtomLmax[iac]);
        std::memcpy(dp.AtomMatrices_[iac], mats + offsets[gid], 2*nc*nc*sizeof(double));
    }
}

void ref_set_energy(void *h, double Er, double Ei, double dVol) {
    auto &p = ((RefPlan*)h)->p;
    green_function::update_energy_parameter(p, std::complex<double>(Er, Ei), dVol, 0, 1, 1.0);
}

void ref_set_kpoint(void *h, const double *k) {
    auto &p = ((RefPlan*)h)->p;
    green_function::update_phases(p, k, 0, 1);
}

// y = (H - E S) x  via the reference's action_t<double,R1C2=2,Noco=1>::multiply
double ref_action_f64(void *h, double *y, const double *x) {
    auto *rp = (RefPlan*)h;
    auto &p = rp->p;
    if (!rp->act64) rp->act64 = new green_action::action_t<double,2,1,64>(&p, 0, 0);
    uint32_t const nnzb = p.colindx.size();
    return rp->act64->multiply((double(*)[2][64][64])y, (double const(*)[2][64][64])x,
                               rp->colIndex.data(), nnzb, p.nCols);
}

double ref_action_f32(void *h, float *y, const float *x) {
    auto *rp = (RefPlan*)h;
    auto &p = rp->p;
    if (!rp->act32) rp->act32 = new green_action::action_t<float,2,1,64>(&p, 0, 0);
    uint32_t const nnzb = p.colindx.size();
    return rp->act32->multiply((float(*)[2][64][64])y, (float const(*)[2][64][64])x,
                               rp->colIndex.data(), nnzb, p.nCols);
}

// green_dyadic::get_projection_coefficients (include/green_dyadic.hxx:1062-1088): the atomic
// density matrices Im <p_i|G|p_j> of every plan atom from an FP64 block vector G, concatenated
// [nAtoms][nSHO][nSHO]; returns -1 where the reference refuses (atom images beyond the atoms)
int ref_projection_coefficients(void *h, const double *G, double *out) {
    auto *rp = (RefPlan*)h;
    auto &p = rp->p;
    auto const &dp = p.dyadic_plan;
    if (dp.nAtomImages != dp.nAtoms) return -1;
    auto const res = green_dyadic::get_projection_coefficients<double,2,1>(
        (double const(*)[2][64][64])G, dp, p.rowindx, p.rowCubePos, p.colCubePos, 0);
    size_t off{0};
    for (auto const &m : res) {
        std::memcpy(out + off, m.data(), m.size()*sizeof(double));
        off += m.size();
    }
    return 0;
}

// kinetic_plan::set_phase (src/kinetic_plan.cxx:214-269): phase[2][2] for one direction
double ref_set_phase(double *phase4, double angle) {
    return kinetic_plan::set_phase((double(*)[2])phase4, angle, 'x', 0);
}

// sho_projection::get_sho_prefactors (include/sho_projection.hxx:190-209)
void ref_sho_prefactors(double *out, int numax, double sigma) {
    auto const f = sho_projection::get_sho_prefactors(numax, sigma);
    for (size_t i = 0; i < f.size(); ++i) out[i] = f[i];
}

// energy_contour::get_energy_mesh (src/energy_contour.cxx:139-240): up to cap points E and
// weights w8 as interleaved (re, im) pairs; returns the number of points
int ref_energy_mesh(double *E, double *w8, int cap, double kBT, double eBot, unsigned nBot, unsigned nPar,
                    unsigned nFer, int nPol) {
    std::vector<std::complex<double>> w;
    auto const Ep = energy_contour::get_energy_mesh(w, kBT, eBot, nBot, nPar, nFer, nPol, 0);
    int const n = int(Ep.size());
    for (int i = 0; i < n && i < cap; ++i) {
        E[2*i] = Ep[i].real(); E[2*i + 1] = Ep[i].imag();
        w8[2*i] = w[i].real(); w8[2*i + 1] = w[i].imag();
    }
    return n;
}

// the quadratures of the contour (src/energy_contour.cxx:456, :2156); x, w hold 128 entries
int ref_gauss_legendre(double *x, double *w, unsigned n) { return energy_contour::Gauss_Legendre_quadrature(x, w, n, 0); }
int ref_gauss_fermi_dirac(double *x, double *w, unsigned n) { return energy_contour::Gauss_Fermi_Dirac_quadrature(x, w, n, 0); }

} // extern "C"

// The contour source also holds the integrator, which calls the solver; the solver needs the
// external tfQMRgpu headers and is not built here.  These definitions only satisfy the linker:
// the oracle never constructs a green_solver_t.
green_solver_t::green_solver_t(action_plan_t *, int, int) { std::fprintf(stderr, "oracle: no solver\n"); }
green_solver_t::~green_solver_t() {}
status_t green_solver_t::solve(std::complex<double> *, uint32_t, int, int, int) { return 1; }
