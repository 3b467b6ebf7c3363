// Host plan construction.  Every array must come out bit-identical to the reference's plan,
// so the floating-point expressions that decide membership (truncation sphere, projection
// spheres, source centre) are evaluated in the same order and precision as there; the
// parity tests compare the arrays element by element.
#include "plan.hpp"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>

namespace a43g {

namespace {

inline double sq(double x) { return x*x; }

// flat index into a box n[3], x fastest (include/kinetic_plan.hxx:9-13)
inline size_t flat3(uint32_t const n[3], uint32_t x, uint32_t y, uint32_t z) {
    return (size_t(z)*n[1] + y)*n[0] + x;
}

template <typename T>
std::string fmt(char const *f, T a) { char b[256]; std::snprintf(b, 256, f, a); return b; }

} // namespace

double set_phase(double phase[2][2], double angle) {
    // exp(2 pi i angle) on the left, its conjugate on the right; on the 15-degree grid the
    // values sin(k 15deg) come from exact surds (src/kinetic_plan.cxx:228-250)
    double const arg = 2*3.14159265358979323846*angle;
    double cs = std::cos(arg), sn = std::sin(arg), dev = 0;
    double const a24 = angle*24;
    int const k = int(a24);
    if (a24 == k) {
        double const sh = std::sqrt(0.5), s3 = std::sqrt(3);
        double const T[7] = {0.0, (s3 - 1)*sh*.5, .5, sh, s3*.5, (s3 + 1)*sh*.5, 1.0};
        int const k24 = ((k % 24) + 24) % 24;
        int const q = k24/6, r = k24 % 6;
        int const is = (q & 1) ? 6 - r : r;
        sn = ((q < 2) ? 1 : -1)*T[is];
        cs = ((q == 1 || q == 2) ? -1 : 1)*T[6 - is];
        dev = std::max(std::abs(cs - std::cos(arg)), std::abs(sn - std::sin(arg)));
    }
    phase[0][0] = cs; phase[0][1] =  sn;
    phase[1][0] = cs; phase[1][1] = -sn;
    return dev;
}

void sho_prefactors(double *out, int numax, double sigma) {
    auto f1 = [sigma](int nu) {
        double fact = 1; for (int i = 2; i <= nu; ++i) fact *= i;
        return std::sqrt(double(1ull << nu)/(fact*std::sqrt(3.14159265358979323846)*sigma));
    };
    int i = 0;
    for (int nz = 0; nz <= numax; ++nz)
        for (int ny = 0; ny <= numax - nz; ++ny)
            for (int nx = 0; nx <= numax - nz - ny; ++nx)
                out[i++] = f1(nx)*f1(ny)*f1(nz);
}

std::string GreenPlan::build(Geometry const &g, ImageRowsFn image_rows) {
    geo = g;
    constexpr int X = 0, Y = 1, Z = 2;
    for (int d = 0; d < 3; ++d) {
        if (g.ng[d] < 4 || g.ng[d] % 4) return "grid points must be positive multiples of 4";
        if (!(g.hg[d] > 0)) return "grid spacings must be positive";
        if (g.bc[d] < BC_ISOLATED || g.bc[d] > BC_REPEAT) return "boundary condition must be 0..3";
        n_blocks[d] = g.ng[d] >> 2;
        bc[d] = g.bc[d];
    }
    if (g.xyzZinso.size() % 8) return "atom list must have 8 entries per atom";

    // ---- source cubes: a box of sources centred in the cell (src/green_function.cxx:316-347)
    int32_t nsrc[3], off[3];
    for (int d = 0; d < 3; ++d) {
        int const ns = int(g.sources[d]);
        nsrc[d] = (ns < 0) ? int32_t(n_blocks[d]) : std::min(std::max(1, ns), int32_t(n_blocks[d]));
        off[d] = (int32_t(n_blocks[d]) - nsrc[d])/2;
    }
    size_t const nrhs = size_t(nsrc[X])*nsrc[Y]*nsrc[Z];
    // uint16 column indices, and the per-column kernels launch one CTA row per source (CUDA grid y <= 65535)
    if (nrhs > 65535) return "at most 65535 source cubes (uint16 column indices, CUDA grid y limit)";
    nCols = uint32_t(nrhs);
    source_coords.resize(3*nrhs);
    {
        size_t irhs = 0;
        for (int bz = 0; bz < nsrc[Z]; ++bz)
        for (int by = 0; by < nsrc[Y]; ++by)
        for (int bx = 0; bx < nsrc[X]; ++bx, ++irhs) {
            source_coords[3*irhs + X] = (bx + off[X]) % int32_t(n_blocks[X]);
            source_coords[3*irhs + Y] = (by + off[Y]) % int32_t(n_blocks[Y]);
            source_coords[3*irhs + Z] = (bz + off[Z]) % int32_t(n_blocks[Z]);
        }
    }

    // ---- source extent and distance of the sources from their centre (:424-466)
    int32_t smin[3] = {1 << 21, 1 << 21, 1 << 21}, smax[3] = {-(1 << 21), -(1 << 21), -(1 << 21)};
    for (size_t i = 0; i < nrhs; ++i)
        for (int d = 0; d < 3; ++d) {
            smin[d] = std::min(smin[d], source_coords[3*i + d]);
            smax[d] = std::max(smax[d], source_coords[3*i + d]);
        }
    {
        double centre[3];
        for (int d = 0; d < 3; ++d) centre[d] = (((smin[d] + smax[d])*0.5)*4 + 2)*g.hg[d];
        double max_d2c = 0;
        for (size_t i = 0; i < nrhs; ++i) {
            double d2c = 0;
            for (int d = 0; d < 3; ++d) d2c += sq((source_coords[3*i + d]*4 + 2)*g.hg[d] - centre[d]);
            max_d2c = std::max(max_d2c, d2c);
        }
        max_distance_from_center = std::sqrt(max_d2c);
    }

    // ---- truncation sphere: effective spacings and boundary conditions (:490-536)
    double const rtrunc = std::max(0., g.r_trunc);
    for (int d = 0; d < 3; ++d) {
        h_trunc[d] = g.hg[d];
        if (g.r_trunc >= 0 && BC_PERIODIC == bc[d]) {
            if (2*rtrunc > h_trunc[d]*g.ng[d]) h_trunc[d] = 0;   // sphere does not fit: no truncation
            else bc[d] = BC_WRAP;                               // fits: wrap like vacuum
        }
    }
    r_block_circumscribing_sphere = 0.5*(4 - 1)*std::sqrt(sq(g.hg[X]) + sq(g.hg[Y]) + sq(g.hg[Z]));
    double const rbcs = r_block_circumscribing_sphere;
    double const r_plus = rtrunc + 2*rbcs;
    double const r_minus = std::max(0., rtrunc - 2*rbcs);
    (void)r_minus;

    int32_t itr[3], tmin[3], tmax[3];
    uint32_t tnum[3];
    for (int d = 0; d < 3; ++d) {
        int32_t const nbox = int32_t(n_blocks[d]) - 1;
        itr[d] = (h_trunc[d] > 0) ? int32_t(std::floor(r_plus/(4*h_trunc[d]))) : nbox;
        if (BC_PERIODIC == bc[d]) itr[d] = std::min(itr[d], nbox);
        tmin[d] = smin[d] - itr[d];
        tmax[d] = smax[d] + itr[d];
        if (BC_ISOLATED == bc[d] || BC_PERIODIC == bc[d]) {
            tmin[d] = std::max(tmin[d], 0);
            tmax[d] = std::min(tmax[d], nbox);
        }
        tnum[d] = uint32_t(std::max(0, tmax[d] + 1 - tmin[d]));
    }
    size_t const nbox3 = size_t(tnum[Z])*tnum[Y]*tnum[X];
    if (0 == nbox3) return "empty target box";

    // ---- block sparsity: a target cube belongs to source i if any grid-point pair is closer
    //      than r_trunc, tested at 8 (far) or 27 (near) corner offsets (:580-694)
    double const r2trunc = sq(rtrunc), r2plus = sq(r_plus), r2circ = sq(rbcs*3);
    // the test depends on the offset (bx, by, bz) from the source only: evaluated once per offset
    // of the box [-itr, itr]^3 (the reference repeats it for every source)
    uint32_t const nof[3] = {uint32_t(2*itr[X] + 1), uint32_t(2*itr[Y] + 1), uint32_t(2*itr[Z] + 1)};
    std::vector<uint8_t> inside(size_t(nof[X])*nof[Y]*nof[Z], 0);
    for (int32_t bz = -itr[Z]; bz <= itr[Z]; ++bz)
    for (int32_t by = -itr[Y]; by <= itr[Y]; ++by)
    for (int32_t bx = -itr[X]; bx <= itr[X]; ++bx) {
        double const d2 = sq(bx*4*h_trunc[X]) + sq(by*4*h_trunc[Y]) + sq(bz*4*h_trunc[Z]);
        int nin = 0;
        if (d2 < r2plus) {
            int const far = (d2 > r2circ);
            int const step = 3 + 3*far;
            for (int iz = -3; iz <= 3; iz += step) {
                double const d2z = sq((bz*4 + iz)*h_trunc[Z]);
                for (int iy = -3; iy <= 3; iy += step) {
                    double const d2yz = sq((by*4 + iy)*h_trunc[Y]) + d2z;
                    for (int ix = -3; ix <= 3; ix += step) {
                        double const d2xyz = sq((bx*4 + ix)*h_trunc[X]) + d2yz;
                        nin += (d2xyz < r2trunc);
                    }
                }
            }
        }
        inside[flat3(nof, uint32_t(bx + itr[X]), uint32_t(by + itr[Y]), uint32_t(bz + itr[Z]))] = (nin > 0);
    }
    std::vector<std::vector<uint16_t>> cols_of(nbox3);
    std::vector<std::vector<bool>> pattern(nrhs, std::vector<bool>(nbox3, false));
    std::vector<int32_t> diag_tag(nbox3, -1);
    for (size_t irhs = 0; irhs < nrhs; ++irhs) {
        int32_t const *sc = &source_coords[3*irhs];
        int32_t bfirst[3], blast[3];
        for (int d = 0; d < 3; ++d) {
            if (BC_ISOLATED == bc[d] || BC_PERIODIC == bc[d]) {
                bfirst[d] = std::max(-itr[d], tmin[d] - sc[d]);
                blast[d]  = std::min( itr[d], tmax[d] - sc[d]);
            } else {
                bfirst[d] = -itr[d];
                blast[d]  =  itr[d];
            }
        }
        for (int32_t bz = bfirst[Z]; bz <= blast[Z]; ++bz)
        for (int32_t by = bfirst[Y]; by <= blast[Y]; ++by)
        for (int32_t bx = bfirst[X]; bx <= blast[X]; ++bx) {
            if (inside[flat3(nof, uint32_t(bx + itr[X]), uint32_t(by + itr[Y]), uint32_t(bz + itr[Z]))]) {
                uint32_t const ix = uint32_t(sc[X] + bx - tmin[X]);
                uint32_t const iy = uint32_t(sc[Y] + by - tmin[Y]);
                uint32_t const iz = uint32_t(sc[Z] + bz - tmin[Z]);
                size_t const idx3 = flat3(tnum, ix, iy, iz);
                if (pattern[irhs][idx3]) return "target cube hit twice by one source";
                pattern[irhs][idx3] = true;
                cols_of[idx3].push_back(uint16_t(irhs));
                if (0 == bx && 0 == by && 0 == bz) diag_tag[idx3] = int32_t(irhs);
            }
        }
    }

    // ---- rows: non-empty target cubes in z,y,x order (:840-944)
    size_t nnz = 0; nRows = 0;
    for (size_t i = 0; i < nbox3; ++i) { nnz += cols_of[i].size(); nRows += !cols_of[i].empty(); }
    if (nnz >= (1ull << 32)) return "too many blocks";
    rowstart.assign(nRows + 1, 0);
    colindx.resize(nnz); rowindx.resize(nnz); veff_index.assign(nnz, -1);
    target_minus_source.assign(4*nnz, 0);
    rowCubePos.assign(4*size_t(nRows), 0.f);
    colCubePos.assign(4*size_t(nCols), 0.f);
    subset.assign(nCols, 0);
    for (size_t i = 0; i < nrhs; ++i)
        for (int d = 0; d < 3; ++d) colCubePos[4*i + d] = float(source_coords[3*i + d] - n_blocks[d]*0.5);
    std::vector<int32_t> row_of(nbox3, -1);
    {
        uint32_t iRow = 0;
        for (uint32_t z = 0; z < tnum[Z]; ++z)
        for (uint32_t y = 0; y < tnum[Y]; ++y)
        for (uint32_t x = 0; x < tnum[X]; ++x) {
            size_t const idx3 = flat3(tnum, x, y, z);
            auto const &cl = cols_of[idx3];
            if (cl.empty()) continue;
            row_of[idx3] = int32_t(iRow);
            uint32_t const r0 = rowstart[iRow];
            rowstart[iRow + 1] = r0 + uint32_t(cl.size());
            std::copy(cl.begin(), cl.end(), colindx.begin() + r0);
            uint32_t const idx[3] = {x, y, z};
            int32_t gt[3];
            for (int d = 0; d < 3; ++d) {
                gt[d] = int32_t(idx[d]) + tmin[d];
                rowCubePos[4*size_t(iRow) + d] = float(gt[d] - n_blocks[d]*0.5);
            }
            int32_t const ic = diag_tag[idx3];
            if (ic >= 0) {
                for (int d = 0; d < 3; ++d)
                    if (colCubePos[4*size_t(ic) + d] != rowCubePos[4*size_t(iRow) + d]) return "diagonal block mismatch";
                for (uint32_t k = r0; k < rowstart[iRow + 1]; ++k)
                    if (colindx[k] == uint32_t(ic)) { subset[ic] = k; break; }
            }
            // potential given in the unit cell, repeated for periodic/wrap/repeat (:896-922)
            int32_t veff = -1;
            {
                bool given = true;
                int32_t mod[3];
                for (int d = 0; d < 3; ++d) {
                    if (BC_VACUUM == bc[d] || BC_ISOLATED == bc[d])
                        given = given && (gt[d] >= 0 && gt[d] < int32_t(n_blocks[d]));
                    mod[d] = gt[d] % int32_t(n_blocks[d]);
                    mod[d] += (mod[d] < 0)*int32_t(n_blocks[d]);
                }
                if (given) veff = int32_t(flat3(n_blocks, mod[X], mod[Y], mod[Z]));
            }
            for (uint32_t k = r0; k < rowstart[iRow + 1]; ++k) {
                uint32_t const ic2 = colindx[k];
                for (int d = 0; d < 3; ++d)
                    target_minus_source[4*size_t(k) + d] = int16_t(double(rowCubePos[4*size_t(iRow) + d]) - double(colCubePos[4*size_t(ic2) + d]));
                rowindx[k] = iRow;
                veff_index[k] = veff;
            }
            ++iRow;
        }
    }

    // ---- finite-difference lists (src/kinetic_plan.cxx:92-209 and :304-322)
    auto find_block = [&](uint32_t x, uint32_t y, uint32_t z, uint32_t irhs) -> int64_t {
        int32_t const r = row_of[flat3(tnum, x, y, z)];
        if (r < 0) return -1;
        for (uint32_t k = rowstart[r]; k < rowstart[r + 1]; ++k) if (colindx[k] == irhs) return k;
        return -1;
    };
    for (int dd = 0; dd < 3; ++dd) {
        auto &K = kinetic[dd];
        K.start.assign(1, 0); K.entry.clear();
        uint32_t num[3] = {tnum[X], tnum[Y], tnum[Z]};
        uint32_t const ndd = num[dd];
        num[dd] = 1;
        uint32_t const periodicity = (BC_PERIODIC == bc[dd]) ? n_blocks[dd] : 0;
        std::vector<int32_t> list;
        for (size_t irhs = 0; irhs < nrhs; ++irhs) {
            for (uint32_t iz = 0; iz < num[Z]; ++iz)
            for (uint32_t iy = 0; iy < num[Y]; ++iy)
            for (uint32_t ix = 0; ix < num[X]; ++ix) {
                uint32_t idx[3] = {ix, iy, iz};
                list.clear();
                int32_t first = -1, last = -1;
                for (uint32_t id = 0; id < ndd; ++id) {
                    idx[dd] = id;
                    if (!pattern[irhs][flat3(tnum, idx[X], idx[Y], idx[Z])]) continue;
                    int64_t const b = find_block(idx[X], idx[Y], idx[Z], uint32_t(irhs));
                    if (b < 0) return "sparsity pattern inconsistent with rows";
                    if (list.empty()) { list.assign(kNhalo, kCubeIsZero); first = int32_t(id); }
                    list.push_back(int32_t(b) + kCubeExists);
                    last = int32_t(id);
                }
                if (list.size() <= size_t(kNhalo)) continue;
                size_t const len = list.size();
                list.resize(len + kNhalo, kCubeIsZero);
                if (periodicity) {
                    if (uint32_t(last + 1 - first) != periodicity) return "periodic line is incomplete";
                    for (int side = 0; side < 2; ++side) {
                        for (int ih = 0; ih < kNhalo; ++ih) {
                            int32_t const jd = side ? (last - int32_t(periodicity) + ih + 1)
                                                    : (first + int32_t(periodicity) + ih - kNhalo);
                            if (jd < 0 || jd >= int32_t(ndd)) continue;
                            uint32_t jdx[3] = {idx[X], idx[Y], idx[Z]};
                            jdx[dd] = uint32_t(jd);
                            if (!pattern[irhs][flat3(tnum, jdx[X], jdx[Y], jdx[Z])]) continue;
                            int64_t const b = find_block(jdx[X], jdx[Y], jdx[Z], uint32_t(irhs));
                            if (b >= 0) list[ih + side*len] = kCubeNeedsPhase*(int32_t(b) + kCubeExists);
                        }
                    }
                }
                K.entry.insert(K.entry.end(), list.begin(), list.end());
                K.start.push_back(uint32_t(K.entry.size()));
            }
        }
        int32_t fd = g.nFD;
        if (periodicity && fd > 4) fd = 4;   // Bloch phases only with the 9-point stencil
        K.FD_range = fd;
        K.prefactor = -0.5*1.0/(g.hg[dd]*g.hg[dd]);
    }
    for (int dd = 0; dd < 3; ++dd) set_phase(phase[dd], 0.0);

    // ---- dyadic plan: atom images whose projection sphere touches a target cube
    //      (src/dyadic_plan.cxx:188-583)
    double const cell[3] = {n_blocks[X]*4*g.hg[X], n_blocks[Y]*4*g.hg[Y], n_blocks[Z]*4*g.hg[Z]};
    for (int d = 0; d < 3; ++d) grid_spacing_dyadic[d] = g.hg[d];
    grid_spacing_dyadic[3] = g.proj_radius;
    double const r_proj = g.proj_radius;
    int32_t const natoms = int32_t(g.xyzZinso.size()/8);
    double max_sigma = 0;
    for (int32_t ia = 0; ia < natoms; ++ia) max_sigma = std::max(max_sigma, g.xyzZinso[ia*8 + 6]);
    for (int32_t ia = 0; ia < natoms; ++ia) if (!(g.xyzZinso[ia*8 + 6] > 0)) return "sigma must be positive";
    double const radius = g.r_trunc + max_distance_from_center + 2*max_sigma*r_proj + 2*rbcs;
    int nimg[3] = {0, 0, 0}, ncpy[3] = {0, 0, 0};
    uint32_t nimages = 1, ncopies = 1;
    for (int d = 0; d < 3; ++d) {
        int const nmx = int(std::max(0., std::ceil(radius/cell[d])));
        if (BC_PERIODIC == bc[d]) nimg[d] = nmx;
        else if (BC_REPEAT == bc[d]) ncpy[d] = nmx;
        else if (BC_WRAP == bc[d]) ncpy[d] = 1;
        nimages *= uint32_t(2*nimg[d] + 1);
        ncopies *= uint32_t(2*ncpy[d] + 1);
    }
    size_t const nAtomCopies = size_t(natoms)*ncopies;

    // every atom copy in every periodic image, in the order of the reference's loops
    struct ImageInfo { double pos[3]; size_t iaa; int32_t ia; int8_t shift[3]; };
    std::vector<ImageInfo> cand;
    std::vector<double> cand_pos, cand_r2p, cand_r2p_plus;
    for (int zi = -nimg[Z]; zi <= nimg[Z]; ++zi)
    for (int yi = -nimg[Y]; yi <= nimg[Y]; ++yi)
    for (int xi = -nimg[X]; xi <= nimg[X]; ++xi) {
        int const ishift[3] = {xi, yi, zi};
        size_t iaa = 0;
        for (int32_t ia = 0; ia < natoms; ++ia) {
            double const sigma = g.xyzZinso[ia*8 + 6];
            double const rp = r_proj*sigma;
            double const r2p = sq(rp), r2p_plus = sq(rp + rbcs);
            for (int zc = -ncpy[Z]; zc <= ncpy[Z]; ++zc)
            for (int yc = -ncpy[Y]; yc <= ncpy[Y]; ++yc)
            for (int xc = -ncpy[X]; xc <= ncpy[X]; ++xc, ++iaa) {
                int const cshift[3] = {xc, yc, zc};
                ImageInfo im;
                for (int d = 0; d < 3; ++d) {
                    im.pos[d] = g.xyzZinso[ia*8 + d] + (ishift[d] + cshift[d])*cell[d];
                    im.shift[d] = int8_t(ishift[d]);
                    cand_pos.push_back(im.pos[d]);
                }
                im.iaa = iaa; im.ia = ia;
                cand.push_back(im);
                cand_r2p.push_back(r2p); cand_r2p_plus.push_back(r2p_plus);
            }
        }
    }
    // target rows whose cube has a corner point inside the projection sphere of each candidate
    std::vector<std::vector<uint32_t>> hits(cand.size());
    if (image_rows && !cand.empty() && nRows > 0) {
        ImageRowsTask t;
        t.ncand = cand.size(); t.pos = cand_pos.data(); t.r2p = cand_r2p.data(); t.r2p_plus = cand_r2p_plus.data();
        t.nRows = nRows; t.rowCubePos = rowCubePos.data();
        for (int d = 0; d < 3; ++d) t.hg[d] = g.hg[d];
        std::string const e = image_rows(t, hits);
        if (!e.empty()) return e;
    } else {
        for (size_t c = 0; c < cand.size(); ++c) {
            double const *pos = &cand_pos[3*c];
            for (uint32_t ir = 0; ir < nRows; ++ir) {
                float const *tc = &rowCubePos[4*size_t(ir)];
                double dc2 = 0;
                for (int d = 0; d < 3; ++d) dc2 += sq((tc[d]*4.f + 2.0)*g.hg[d] - pos[d]);
                if (dc2 > cand_r2p_plus[c]) continue;
                double d2c[3][2];
                for (int d = 0; d < 3; ++d)
                    for (int ii = 0; ii < 2; ++ii) d2c[d][ii] = sq((tc[d]*4.0 + ii*3 + 0.5)*g.hg[d] - pos[d]);
                int nin = 0;
                for (int i8 = 0; i8 < 8; ++i8)
                    nin += (d2c[X][i8 & 1] + d2c[Y][(i8 & 2) >> 1] + d2c[Z][i8 >> 2] < cand_r2p[c]);
                if (nin > 0) hits[c].push_back(ir);
            }
        }
    }
    std::vector<ImageInfo> images;
    std::vector<std::vector<uint32_t>> cubes;   // target rows hit by each contributing image
    std::vector<bool> copy_contributes(nAtomCopies, false);
    AtomImageStarts.assign(1, 0);
    for (size_t c = 0; c < cand.size(); ++c) {
        if (hits[c].empty()) continue;
        copy_contributes[cand[c].iaa] = true;
        images.push_back(cand[c]);
        cubes.push_back(std::move(hits[c]));
        AtomImageStarts.push_back(AtomImageStarts.back() + uint32_t(nsho(int(g.xyzZinso[cand[c].ia*8 + 5]))));
    }
    nAtomImages = uint32_t(images.size());
    uint32_t const nAI = nAtomImages;

    // projection (per source) and addition (per block) sparsity
    std::vector<std::vector<std::vector<uint32_t>>> prj(nrhs, std::vector<std::vector<uint32_t>>(nAI));
    std::vector<std::vector<uint32_t>> add(nnz);
    for (uint32_t a = 0; a < nAI; ++a)
        for (uint32_t ir : cubes[a])
            for (uint32_t k = rowstart[ir]; k < rowstart[ir + 1]; ++k) {
                prj[colindx[k]][a].push_back(k);
                add[k].push_back(a);
            }
    auto to_csr = [](std::vector<std::vector<uint32_t>> const &rows) {
        Csr c; c.start.assign(1, 0);
        for (auto const &r : rows) { c.col.insert(c.col.end(), r.begin(), r.end()); c.start.push_back(uint32_t(c.col.size())); }
        return c;
    };
    SHOadd = to_csr(add);
    SHOprj.resize(nrhs);
    for (size_t s = 0; s < nrhs; ++s) SHOprj[s] = to_csr(prj[s]);

    // projector tables per (image, row) slot (include/green_dyadic.hxx:33-107 evaluates them
    // per (image, block) on the fly; here once, on the host, in the CPU order of operations)
    img_rows = to_csr(cubes);
    table_lmax = -1;
    for (auto const &im : images) table_lmax = std::max(table_lmax, int(g.xyzZinso[im.ia*8 + 5]));
    {
        int const nt = (table_lmax + 1)*12;
        size_t const nslots = img_rows.nnz();
        slot_H.assign(nslots*size_t(std::max(nt, 1)), 0.0);
        slot_mask.assign(nslots, 0);
        double const R2 = g.proj_radius*g.proj_radius;
        float const R2f = float(R2);
        for (uint32_t a = 0; a < nAI; ++a) {
            auto const &im = images[a];
            int const lmax = int(g.xyzZinso[im.ia*8 + 5]);
            double const isq = 1./std::sqrt(g.xyzZinso[im.ia*8 + 6]);   // stored as 1/sqrt(sigma)
            double const sinv = isq*isq;
            for (uint32_t k = img_rows.start[a]; k < img_rows.start[a + 1]; ++k) {
                float const *tc = &rowCubePos[4*size_t(img_rows.col[k])];
                double *H = &slot_H[size_t(k)*nt];
                float xi2[3][4];
                for (int d = 0; d < 3; ++d)
                    for (int i4 = 0; i4 < 4; ++i4) {
                        double const xi = sinv*((double(tc[d])*4 + i4 + 0.5)*g.hg[d] - im.pos[d]);
                        double const x2 = xi*xi;
                        xi2[d][i4] = float(x2);
                        double hm = 0, h = (x2 < R2) ? std::exp(-0.5*x2) : 0.0;
                        H[(0*3 + d)*4 + i4] = h;
                        for (int nu = 0; nu < lmax; ++nu) {
                            double const hp = xi*h - 0.5*nu*hm;
                            H[((nu + 1)*3 + d)*4 + i4] = hp;
                            hm = h; h = hp;
                        }
                    }
                uint64_t mask = 0;   // ((xi2_z - R2) + xi2_y) + xi2_x < 0 in float
                for (int z = 0; z < 4; ++z) {
                    float const d2z = xi2[2][z] - R2f;
                    for (int y = 0; y < 4; ++y) {
                        float const d2yz = xi2[1][y] + d2z;
                        for (int x = 0; x < 4; ++x)
                            if (xi2[0][x] + d2yz < 0.f) mask |= 1ull << ((z*4 + y)*4 + x);
                    }
                }
                slot_mask[k] = mask;
            }
        }
        // slot of every projection and addition pair
        prj_slot.clear(); add_slot.assign(SHOadd.nnz(), 0);
        auto slot = [&](uint32_t a, uint32_t row) -> uint32_t {
            // rows of one image are sorted ascending (target rows scanned in order)
            auto const b = img_rows.col.begin() + img_rows.start[a], e = img_rows.col.begin() + img_rows.start[a + 1];
            return uint32_t(std::lower_bound(b, e, row) - img_rows.col.begin());
        };
        for (size_t s = 0; s < nrhs; ++s)
            for (uint32_t a = 0; a < nAI; ++a)
                for (uint32_t k = SHOprj[s].start[a]; k < SHOprj[s].start[a + 1]; ++k)
                    prj_slot.push_back(slot(a, rowindx[SHOprj[s].col[k]]));
        for (uint32_t b = 0; b < nnz; ++b)
            for (uint32_t k = SHOadd.start[b]; k < SHOadd.start[b + 1]; ++k)
                add_slot[k] = slot(SHOadd.col[k], rowindx[b]);
    }

    // contributing atom copies, their matrices and the image -> atom relation
    std::vector<int32_t> iac_of_iaa(nAtomCopies, -1);
    global_atom_ids.clear();
    for (size_t iaa = 0; iaa < nAtomCopies; ++iaa) {
        if (!copy_contributes[iaa]) continue;
        iac_of_iaa[iaa] = int32_t(global_atom_ids.size());
        global_atom_ids.push_back(int64_t(g.xyzZinso[(iaa/ncopies)*8 + 4]));
    }
    nAtoms = uint32_t(global_atom_ids.size());
    AtomImageIndex.resize(nAI); AtomImagePos.resize(4*size_t(nAI)); AtomImageLmax.resize(nAI);
    AtomImageShift.assign(4*size_t(nAI), 0); AtomImagePhase.assign(4*size_t(nAI), 0.0);
    std::vector<std::vector<uint32_t>> sum(nAtoms);
    for (uint32_t a = 0; a < nAI; ++a) {
        auto const &im = images[a];
        double const sigma = g.xyzZinso[im.ia*8 + 6];
        int32_t const iac = iac_of_iaa[im.iaa];
        AtomImageIndex[a] = uint32_t(iac);
        for (int d = 0; d < 3; ++d) { AtomImagePos[4*a + d] = im.pos[d]; AtomImageShift[4*a + d] = im.shift[d]; }
        AtomImagePos[4*a + 3] = 1./std::sqrt(sigma);
        AtomImageLmax[a] = int8_t(int(g.xyzZinso[im.ia*8 + 5]));
        AtomImagePhase[4*a] = 1.0;
        sum[iac].push_back(a);
    }
    SHOsum = to_csr(sum);
    AtomStarts.assign(1, 0); AtomLmax.resize(nAtoms); AtomSigma.resize(nAtoms);
    AtomMatOffset.assign(1, 0);
    for (uint32_t iac = 0; iac < nAtoms; ++iac) {
        int64_t const id = global_atom_ids[iac];   // the atom id doubles as its index (src/dyadic_plan.cxx:556-558)
        if (id < 0 || id >= natoms) return "atom ids must be the atom indices 0..natoms-1";
        int const numax = int(g.xyzZinso[id*8 + 5]);
        AtomSigma[iac] = g.xyzZinso[id*8 + 6];
        AtomLmax[iac] = int8_t(numax);
        int const nc = nsho(numax);
        AtomStarts.push_back(AtomStarts.back() + uint32_t(nc));
        AtomMatOffset.push_back(AtomMatOffset.back() + uint32_t(2*nc*nc));
    }
    AtomMatricesIn.assign(AtomMatOffset.back(), 0.0);
    AtomMatrices.assign(AtomMatOffset.back(), 0.0);
    for (uint32_t iac = 0; iac < nAtoms; ++iac)
        for (uint32_t k = SHOsum.start[iac]; k < SHOsum.start[iac + 1]; ++k)
            if (AtomImageLmax[SHOsum.col[k]] != AtomLmax[iac]) return "image and atom basis sizes differ";

    Vcell.assign(ncells()*64, 0.0);
    E_re = E_im = 0;
    return "";
}

std::string GreenPlan::set_potential_grid(double const *V) {
    uint32_t const nx = geo.ng[0], ny = geo.ng[1];
    for (uint32_t bz = 0; bz < n_blocks[2]; ++bz)
    for (uint32_t by = 0; by < n_blocks[1]; ++by)
    for (uint32_t bx = 0; bx < n_blocks[0]; ++bx) {
        size_t const c = flat3(n_blocks, bx, by, bz);
        for (int i = 0; i < 64; ++i) {
            size_t const ix = bx*4 + (i & 3), iy = by*4 + ((i >> 2) & 3), iz = bz*4 + (i >> 4);
            Vcell[c*64 + i] = V[(iz*ny + iy)*nx + ix];
        }
    }
    return "";
}

std::string GreenPlan::set_potential_cells(double const *Vc) {
    std::memcpy(Vcell.data(), Vc, Vcell.size()*sizeof(double));
    return "";
}

std::string GreenPlan::set_atom_matrices(double const *mats, int64_t const *offsets, int64_t natoms) {
    for (uint32_t iac = 0; iac < nAtoms; ++iac) {
        int64_t const id = global_atom_ids[iac];
        if (id < 0 || id >= natoms) return "atom id out of range";
        int const nc = nsho(AtomLmax[iac]);
        std::memcpy(&AtomMatricesIn[AtomMatOffset[iac]], mats + offsets[id], 2*size_t(nc)*nc*sizeof(double));
    }
    return "";
}

void GreenPlan::set_energy(double Er, double Ei, double dVol, double scale_H) {
    E_re = Er; E_im = Ei;
    for (uint32_t iac = 0; iac < nAtoms; ++iac) {
        int const nc = nsho(AtomLmax[iac]);
        double const *hmt = &AtomMatricesIn[AtomMatOffset[iac]];
        double const *ovl = hmt + nc*nc;
        double *m = &AtomMatrices[AtomMatOffset[iac]];
        for (int ij = 0; ij < nc*nc; ++ij) {
            m[ij]         = (scale_H*hmt[ij] - Er*ovl[ij])*dVol;
            m[ij + nc*nc] = (              - Ei*ovl[ij])*dVol;
        }
    }
}

std::string GreenPlan::set_kpoint(double const k[3]) {
    for (int d = 0; d < 3; ++d) {
        if (!(std::abs(k[d]) < 0.503)) return "k-point components must be below 0.503 (units of 2 pi / cell)";
        set_phase(phase[d], k[d]);
    }
    // phase of an image = product over directions of phase^shift (left phase for shift >= 0)
    auto ipow = [](std::complex<double> x, unsigned n) {
        std::complex<double> r(1, 0);
        while (n) { if (n & 1) r *= x; n >>= 1; x *= x; }
        return r;
    };
    for (uint32_t a = 0; a < nAtomImages; ++a) {
        std::complex<double> ph(1, 0);
        for (int d = 0; d < 3; ++d) {
            int const s = AtomImageShift[4*a + d];
            std::complex<double> const fwd(phase[d][0][0], phase[d][0][1]), bwd(phase[d][1][0], phase[d][1][1]);
            ph *= (s >= 0) ? ipow(fwd, unsigned(s)) : ipow(bwd, unsigned(-s));
        }
        AtomImagePhase[4*a + 0] = ph.real(); AtomImagePhase[4*a + 1] = ph.imag();
        AtomImagePhase[4*a + 2] = 0; AtomImagePhase[4*a + 3] = 0;
    }
    return "";
}

// d/dR H_nu(xi) = -(1/sigma) (nu H_{nu-1}(xi) - xi H_nu(xi)) with xi = (r - R)/sigma, because the
// unnormalized Hermite-Gauss functions H_nu = h_nu exp(-xi^2/2) have h_nu' = nu h_{nu-1}; the
// points and the cut-off are those of slot_H (the 1D functions vanish outside the radius)
std::vector<double> GreenPlan::position_derivative_tables(int dir) const {
    std::vector<double> T(slot_H);
    if (table_lmax < 0 || dir < 0 || dir > 2) return T;
    int const nt = (table_lmax + 1)*12;
    for (uint32_t a = 0; a < nAtomImages; ++a) {
        int const lmax = AtomImageLmax[a];
        double const isq = AtomImagePos[4*size_t(a) + 3], sinv = isq*isq;
        for (uint32_t k = img_rows.start[a]; k < img_rows.start[a + 1]; ++k) {
            float const *tc = &rowCubePos[4*size_t(img_rows.col[k])];
            double const *H = &slot_H[size_t(k)*nt];
            double *D = &T[size_t(k)*nt];
            for (int i4 = 0; i4 < 4; ++i4) {
                double const xi = sinv*((double(tc[dir])*4 + i4 + 0.5)*grid_spacing_dyadic[dir] - AtomImagePos[4*size_t(a) + dir]);
                for (int nu = 0; nu <= lmax; ++nu) {
                    double const hn = H[(nu*3 + dir)*4 + i4];
                    double const hm = (nu > 0) ? H[((nu - 1)*3 + dir)*4 + i4] : 0.0;
                    D[(nu*3 + dir)*4 + i4] = -sinv*(nu*hm - xi*hn);
                }
            }
        }
    }
    return T;
}

} // namespace a43g

namespace a43g {

// Batch plan: npairs copies of the one-pair plan `one`.  Every row r keeps its target cube; its
// blocks are those of `one` repeated once per pair, pair-major, so the block of pair p at position
// i of row r is  npairs*rowstart[r] + p*len_r + i  and its source column is  c + p*nsrc.  Every
// array indexed by block or source is remapped accordingly; the atom images, projector tables and
// potential are shared by all pairs.
std::string GreenPlan::replicate(GreenPlan const &one, uint32_t P) {
    if (P < 1) return "at least one (energy, k-point) pair";
    if (one.npairs != 1) return "replicate needs a one-pair plan";
    size_t const nsrc = one.nCols;
    if (size_t(P)*nsrc > 65535) return "at most 65535 source cubes in a batch (uint16 column indices)";
    *this = one;
    npairs = P; nsrc_pair = uint32_t(nsrc);
    nCols = uint32_t(P*nsrc);
    size_t const nnzb1 = one.nnzb(), nnzb = nnzb1*P;
    // block map
    std::vector<uint32_t> map(nnzb1*P);
    rowstart.assign(one.nRows + 1, 0);
    colindx.resize(nnzb); rowindx.resize(nnzb); veff_index.resize(nnzb);
    target_minus_source.resize(4*nnzb);
    for (uint32_t r = 0; r < one.nRows; ++r) {
        uint32_t const b0 = one.rowstart[r], len = one.rowstart[r + 1] - b0;
        rowstart[r] = uint32_t(P*size_t(b0));
        for (uint32_t p = 0; p < P; ++p)
            for (uint32_t i = 0; i < len; ++i) {
                size_t const nb = P*size_t(b0) + size_t(p)*len + i, ob = b0 + i;
                map[size_t(p)*nnzb1 + ob] = uint32_t(nb);
                colindx[nb] = uint16_t(one.colindx[ob] + p*nsrc);
                rowindx[nb] = one.rowindx[ob];
                veff_index[nb] = one.veff_index[ob];
                for (int k = 0; k < 4; ++k) target_minus_source[4*nb + k] = one.target_minus_source[4*ob + k];
            }
    }
    rowstart[one.nRows] = uint32_t(nnzb);
    auto remap = [&](uint32_t p, uint32_t b) { return map[size_t(p)*nnzb1 + b]; };
    subset.resize(nCols); colCubePos.resize(4*size_t(nCols)); source_coords.resize(3*size_t(nCols));
    for (uint32_t p = 0; p < P; ++p)
        for (size_t s = 0; s < nsrc; ++s) {
            subset[p*nsrc + s] = remap(p, one.subset[s]);
            for (int k = 0; k < 4; ++k) colCubePos[4*(p*nsrc + s) + k] = one.colCubePos[4*s + k];
            for (int k = 0; k < 3; ++k) source_coords[3*(p*nsrc + s) + k] = one.source_coords[3*s + k];
        }
    // finite-difference lists: every list of `one` once per pair, entries remapped
    for (int dd = 0; dd < 3; ++dd) {
        auto const &K1 = one.kinetic[dd];
        auto &K = kinetic[dd];
        K.start.assign(1, 0); K.entry.clear();
        K.entry.reserve(K1.entry.size()*P);
        for (uint32_t p = 0; p < P; ++p)
            for (uint32_t il = 0; il < K1.nlists(); ++il) {
                for (uint32_t k = K1.start[il]; k < K1.start[il + 1]; ++k) {
                    int32_t const e = K1.entry[k];
                    if (e > 0) K.entry.push_back(int32_t(remap(p, uint32_t(e - 1))) + 1);
                    else if (e < 0) K.entry.push_back(-(int32_t(remap(p, uint32_t(-e - 1))) + 1));
                    else K.entry.push_back(0);
                }
                K.start.push_back(uint32_t(K.entry.size()));
            }
    }
    // projector sparsity: SHOprj per source (columns are blocks), SHOadd per block
    SHOprj.assign(nCols, Csr{});
    prj_slot.clear();
    {
        std::vector<size_t> slot_off(nsrc + 1, 0);
        for (size_t s = 0; s < nsrc; ++s) slot_off[s + 1] = slot_off[s] + one.SHOprj[s].nnz();
        for (uint32_t p = 0; p < P; ++p)
            for (size_t s = 0; s < nsrc; ++s) {
                Csr const &c1 = one.SHOprj[s];
                Csr &c = SHOprj[p*nsrc + s];
                c.start = c1.start;
                c.col.resize(c1.col.size());
                for (size_t k = 0; k < c1.col.size(); ++k) c.col[k] = remap(p, c1.col[k]);
                prj_slot.insert(prj_slot.end(), one.prj_slot.begin() + slot_off[s], one.prj_slot.begin() + slot_off[s + 1]);
            }
    }
    {
        std::vector<uint32_t> inv(nnzb);                 // new block -> old block
        for (uint32_t p = 0; p < P; ++p) for (size_t b = 0; b < nnzb1; ++b) inv[remap(p, uint32_t(b))] = uint32_t(b);
        SHOadd.start.assign(1, 0); SHOadd.col.clear(); add_slot.clear();
        SHOadd.col.reserve(one.SHOadd.nnz()*P); add_slot.reserve(one.SHOadd.nnz()*P);
        for (size_t nb = 0; nb < nnzb; ++nb) {
            uint32_t const ob = inv[nb];
            for (uint32_t k = one.SHOadd.start[ob]; k < one.SHOadd.start[ob + 1]; ++k) {
                SHOadd.col.push_back(one.SHOadd.col[k]);
                add_slot.push_back(one.add_slot[k]);
            }
            SHOadd.start.push_back(uint32_t(SHOadd.col.size()));
        }
    }
    // per-pair values start as copies of the one-pair values
    pair_E.assign(2*size_t(P), 0);
    pair_phase.resize(12*size_t(P));
    pair_img_phase.resize(size_t(P)*AtomImagePhase.size());
    pair_mats.resize(size_t(P)*AtomMatrices.size());
    for (uint32_t p = 0; p < P; ++p) {
        pair_E[2*p] = one.E_re; pair_E[2*p + 1] = one.E_im;
        std::memcpy(&pair_phase[12*size_t(p)], one.phase, sizeof(one.phase));
        std::copy(one.AtomImagePhase.begin(), one.AtomImagePhase.end(), pair_img_phase.begin() + size_t(p)*AtomImagePhase.size());
        std::copy(one.AtomMatrices.begin(), one.AtomMatrices.end(), pair_mats.begin() + size_t(p)*AtomMatrices.size());
    }
    return "";
}

std::string GreenPlan::set_pair(uint32_t p, double Er, double Ei, double dVol, double const k[3]) {
    if (p >= npairs) return "pair index beyond the batch";
    // the one-pair updates on this plan's own arrays, then copied into the pair's slots
    set_energy(Er, Ei, dVol);
    auto const err = set_kpoint(k);
    if (!err.empty()) return err;
    pair_E[2*size_t(p)] = Er; pair_E[2*size_t(p) + 1] = Ei;
    std::memcpy(&pair_phase[12*size_t(p)], phase, sizeof(phase));
    std::copy(AtomImagePhase.begin(), AtomImagePhase.end(), pair_img_phase.begin() + size_t(p)*AtomImagePhase.size());
    std::copy(AtomMatrices.begin(), AtomMatrices.end(), pair_mats.begin() + size_t(p)*AtomMatrices.size());
    return "";
}

} // namespace a43g

namespace a43g {

// The 1D Hermite-Gauss functions and the spherical mask of every (image, source cube) pair,
// evaluated as the slot tables are (the same expressions in the same order) but at the points
// of the source cube: colCubePos instead of rowCubePos.
void GreenPlan::source_tables(std::vector<double> &H, std::vector<uint64_t> &mask) const {
    int const nt = (table_lmax + 1)*12;
    H.assign(size_t(nAtomImages)*nCols*size_t(std::max(nt, 1)), 0.0);
    mask.assign(size_t(nAtomImages)*nCols, 0);
    if (table_lmax < 0) return;
    double const R2 = geo.proj_radius*geo.proj_radius;
    float const R2f = float(R2);
    for (uint32_t a = 0; a < nAtomImages; ++a) {
        int const lmax = AtomImageLmax[a];
        double const isq = AtomImagePos[4*size_t(a) + 3];          // 1/sqrt(sigma)
        double const sinv = isq*isq;
        double const pos[3] = {AtomImagePos[4*size_t(a)], AtomImagePos[4*size_t(a) + 1], AtomImagePos[4*size_t(a) + 2]};
        for (uint32_t s = 0; s < nCols; ++s) {
            float const *tc = &colCubePos[4*size_t(s)];
            double *h1 = &H[(size_t(a)*nCols + s)*nt];
            float xi2[3][4];
            for (int d = 0; d < 3; ++d)
                for (int i4 = 0; i4 < 4; ++i4) {
                    double const xi = sinv*((double(tc[d])*4 + i4 + 0.5)*geo.hg[d] - pos[d]);
                    double const x2 = xi*xi;
                    xi2[d][i4] = float(x2);
                    double hm = 0, h = (x2 < R2) ? std::exp(-0.5*x2) : 0.0;
                    h1[(0*3 + d)*4 + i4] = h;
                    for (int nu = 0; nu < lmax; ++nu) {
                        double const hp = xi*h - 0.5*nu*hm;
                        h1[((nu + 1)*3 + d)*4 + i4] = hp;
                        hm = h; h = hp;
                    }
                }
            uint64_t m = 0;
            for (int z = 0; z < 4; ++z) {
                float const d2z = xi2[2][z] - R2f;
                for (int y = 0; y < 4; ++y) {
                    float const d2yz = xi2[1][y] + d2z;
                    for (int x = 0; x < 4; ++x)
                        if (xi2[0][x] + d2yz < 0.f) m |= 1ull << ((z*4 + y)*4 + x);
                }
            }
            mask[size_t(a)*nCols + s] = m;
        }
    }
}

} // namespace a43g
