// Host-side plan of the block-sparse Green-function action.
//
// Built by GreenPlan::build (plan_builder.cpp), which restates the reference's plan
// construction so that every array is bit-identical to it:
//   src/green_function.cxx:357-1068 construct_Green_function (sources, truncation sphere,
//                                   block-sparse rows, potential indirection, diagonal subset)
//   src/kinetic_plan.cxx:38-210     finite-difference lists per direction
//   src/dyadic_plan.cxx:159-583     atom images and the projector sparsity
// The device copy of a plan lives in device_plan.cuh.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace a43g {

// boundary conditions (include/boundary_condition.hxx:17-39)
enum : int8_t { BC_ISOLATED = 0, BC_PERIODIC = 1, BC_VACUUM = 2, BC_REPEAT = 3, BC_WRAP = 5 };

// finite-difference list markers (include/kinetic_plan.hxx:19-23)
constexpr int     kNhalo        = 4;
constexpr int32_t kCubeExists   = 1;
constexpr int32_t kCubeIsZero   = 0;
constexpr int32_t kCubeNeedsPhase = -1;

inline int nsho(int numax) { return ((1 + numax)*(2 + numax)*(3 + numax))/6; }

struct Csr {                       // compressed rows
    std::vector<uint32_t> start;   // [nrows + 1]
    std::vector<uint32_t> col;     // [nnz]
    uint32_t nrows() const { return start.empty() ? 0u : uint32_t(start.size() - 1); }
    uint32_t nnz() const { return start.empty() ? 0u : start.back(); }
};

struct Geometry {
    uint32_t ng[3];                // grid points (multiples of 4)
    int8_t   bc[3];                // BC_ISOLATED, BC_PERIODIC, BC_VACUUM, BC_REPEAT
    double   hg[3];                // grid spacings (Bohr)
    double   r_trunc;              // truncation radius (Bohr), < 0: no truncation
    double   sources[3];           // source cubes per direction, < 0: all
    int32_t  nFD;                  // finite-difference range: 4 (8th order) or 8 (16th order)
    double   proj_radius;          // projection radius in units of sigma
    std::vector<double> xyzZinso;  // [natoms*8]: x,y,z (relative to the cell centre), Z, id, numax, sigma, unused
};

struct KineticLists {
    std::vector<uint32_t> start;   // [nlists + 1]
    std::vector<int32_t>  entry;   // inzb+1, 0 (zero cube) or -(inzb+1) (periodic image with phase)
    int32_t FD_range = 0;          // 4 or 8 (< 1: off)
    double  prefactor = 0;         // -1/(2 h^2)
    uint32_t nlists() const { return start.empty() ? 0u : uint32_t(start.size() - 1); }
};

// the projection-sphere test of the dyadic plan for every candidate atom image (position, squared
// projection radius and that radius plus the cube's circumscribing sphere) against every target
// row: hits[c] receives the rows of candidate c in ascending order
struct ImageRowsTask {
    size_t ncand = 0;
    double const *pos = nullptr;               // [ncand][3]
    double const *r2p = nullptr, *r2p_plus = nullptr;   // [ncand]
    uint32_t nRows = 0;
    float const *rowCubePos = nullptr;         // [nRows][4]
    double hg[3] = {0, 0, 0};
};
using ImageRowsFn = std::string (*)(ImageRowsTask const &task, std::vector<std::vector<uint32_t>> &hits);

// the same test on the current CUDA device (plan_device.cu), bit-identical to the host loop
std::string image_rows_on_device(ImageRowsTask const &task, std::vector<std::vector<uint32_t>> &hits);

struct GreenPlan {
    Geometry geo;
    uint32_t n_blocks[3] = {0, 0, 0};
    int8_t   bc[3] = {0, 0, 0};    // effective boundary conditions (periodic may become wrap)
    double   h_trunc[3] = {0, 0, 0};
    double   r_block_circumscribing_sphere = 0;
    double   max_distance_from_center = 0;

    uint32_t nRows = 0, nCols = 0;
    std::vector<uint32_t> rowstart;            // [nRows + 1]
    std::vector<uint16_t> colindx;             // [nnzb]
    std::vector<uint32_t> rowindx;             // [nnzb]
    std::vector<int32_t>  veff_index;          // [nnzb] cell-cube index, -1: no potential
    std::vector<uint32_t> subset;              // [nCols] block index of each diagonal block
    std::vector<float>    rowCubePos;          // [nRows][4]
    std::vector<float>    colCubePos;          // [nCols][4]
    std::vector<int16_t>  target_minus_source; // [nnzb][4]
    std::vector<int32_t>  source_coords;       // [nCols][3] global cube coordinates of the sources

    KineticLists kinetic[3];
    double phase[3][2][2] = {};                // [dd][left,right][re,im]

    // dyadic plan
    uint32_t nAtoms = 0, nAtomImages = 0;
    std::vector<uint32_t> AtomStarts;          // [nAtoms + 1]
    std::vector<int8_t>   AtomLmax;            // [nAtoms]
    std::vector<double>   AtomSigma;           // [nAtoms]
    std::vector<int64_t>  global_atom_ids;     // [nAtoms]
    std::vector<uint32_t> AtomImageIndex;      // [nAI]
    std::vector<uint32_t> AtomImageStarts;     // [nAI + 1]
    std::vector<double>   AtomImagePos;        // [nAI][4]: x,y,z, 1/sqrt(sigma)
    std::vector<int8_t>   AtomImageLmax;       // [nAI]
    std::vector<int8_t>   AtomImageShift;      // [nAI][4]
    std::vector<double>   AtomImagePhase;      // [nAI][4]
    double grid_spacing_dyadic[4] = {0, 0, 0, 0}; // hx, hy, hz, projection radius (sigma units)
    Csr SHOadd;                                // rows: blocks, cols: atom images
    std::vector<Csr> SHOprj;                   // [nCols] rows: atom images, cols: blocks
    Csr SHOsum;                                // rows: atoms, cols: atom images
    // projector tables per (atom image, target row) slot, shared by every source column:
    // 1D Hermite-Gauss functions H[nu][dir][i4] (nu <= lmax_max) and the 64-point spherical mask
    Csr img_rows;                              // rows: atom images, cols: target rows hit (slot = position)
    int table_lmax = -1;                       // nu range of the tables
    std::vector<double>   slot_H;              // [nslots][(table_lmax+1)*12]
    std::vector<uint64_t> slot_mask;           // [nslots]
    std::vector<uint32_t> prj_slot;            // aligned with the concatenated SHOprj columns
    std::vector<uint32_t> add_slot;            // aligned with SHOadd.col
    std::vector<uint32_t> AtomMatOffset;       // [nAtoms + 1] offsets into matrix storage (2*nc*nc each)
    std::vector<double>   AtomMatricesIn;      // per contributing atom: [2][nc][nc] (hmt, ovl) rescaled
    std::vector<double>   AtomMatrices;        // per contributing atom: [2][nc][nc] (re, im) of dVol (H - E S)

    // energy and potential
    double E_re = 0, E_im = 0;
    std::vector<double> Vcell;                 // [ncells][64]

    // batch of independent (energy, k-point) pairs on one geometry (replicate): the sources of
    // pair p are s + p*nsrc_pair, every pair has its own energy, phases and atom matrices
    uint32_t npairs = 1, nsrc_pair = 0;        // nsrc_pair = nCols / npairs
    std::vector<double> pair_E;                // [npairs][2]
    std::vector<double> pair_phase;            // [npairs][3][2][2]
    std::vector<double> pair_img_phase;        // [npairs][nAI][4]
    std::vector<double> pair_mats;             // [npairs][AtomMatrices.size()]

    size_t nnzb() const { return colindx.size(); }
    size_t ncells() const { return size_t(n_blocks[0])*n_blocks[1]*n_blocks[2]; }
    size_t ncoeff_images() const { return AtomImageStarts.empty() ? 0 : AtomImageStarts.back(); }
    size_t ncoeff_atoms() const { return AtomStarts.empty() ? 0 : AtomStarts.back(); }

    // returns an empty string on success, else an error message; image_rows (optional) evaluates
    // the atom-image x target-row test (default: the host loop)
    std::string build(Geometry const &g, ImageRowsFn image_rows = nullptr);
    // potential on the full grid, natural order V[(iz*ng_y + iy)*ng_x + ix]
    std::string set_potential_grid(double const *V);
    // potential already in cell-cube layout [ncells][64]
    std::string set_potential_cells(double const *Vc);
    // per original atom (indexed by atom id): concatenated [2][nc][nc] (hmt, ovl), offsets[natoms]
    std::string set_atom_matrices(double const *mats, int64_t const *offsets, int64_t natoms);
    // update_energy_parameter (src/green_function.cxx:64-109)
    void set_energy(double Er, double Ei, double dVol, double scale_H = 1.0);
    // update_phases (src/green_function.cxx:218-251)
    std::string set_kpoint(double const k[3]);
    // slot_H with the functions of direction dir replaced by their derivative with respect to
    // the atom position (vector-Jacobian products; the reference has no derivatives)
    std::vector<double> position_derivative_tables(int dir) const;
    // projector tables of every (atom image, source cube) pair, in the layout of slot_H and
    // slot_mask (the functions evaluated at the points of the source cube instead of a target
    // cube; green_dyadic::SHOprj_right, include/green_dyadic.hxx:925-1060)
    void source_tables(std::vector<double> &H, std::vector<uint64_t> &mask) const;
    // this plan as npairs copies of the one-pair plan `one` (same geometry, potential and atom
    // matrices; no reference counterpart: the reference solves its (E, k) points one by one)
    std::string replicate(GreenPlan const &one, uint32_t npairs);
    // energy and k-point of pair p of a replicated plan (the one-pair set_energy/set_kpoint)
    std::string set_pair(uint32_t p, double Er, double Ei, double dVol, double const k[3]);
};

// set_phase (src/kinetic_plan.cxx:214-269): returns the deviation of the purified values
double set_phase(double phase[2][2], double angle);

// SHO prefactors sqrt(2^nu/(nu! sqrt(pi) sigma)) products in zyx order (include/sho_projection.hxx:181-209)
void sho_prefactors(double *out, int numax, double sigma);

} // namespace a43g
