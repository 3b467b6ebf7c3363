// The C ABI used from C++, as AngstromCube's own host code would use it: a plan built from a
// geometry (construct_Green_function's inputs), its sizes and two exported arrays, and a grid
// Hamiltonian written and read back.  Needs no GPU.  Prints one JSON line; exit status 0 on
// success.  Usage: plan_from_cxx <scratch file name ending in .xml>
#include "a43g.h"

#include <cstdio>
#include <cstring>
#include <vector>

static int fail(char const *what) {
    std::fprintf(stderr, "%s: %s\n", what, a43g_last_error());
    return 1;
}

int main(int argc, char **argv) {
    if (argc < 2) return 2;
    // periodic 4x4x4-cube cell (16^3 points, h = 0.25 Bohr), one atom at the centre, numax 3
    double const atom[8] = {0.0, 0.0, 0.0, 13, 0, 3, 0.5, 0};
    a43g_geometry_t g;
    std::memset(&g, 0, sizeof(g));
    for (int d = 0; d < 3; ++d) { g.ng[d] = 16; g.bc[d] = 1; g.hg[d] = 0.25; g.sources[d] = 1; }
    g.r_trunc = 3.0; g.nFD = 4; g.proj_radius = 6.0; g.natoms = 1; g.xyzZinso = atom;
    a43g_plan_t *plan = nullptr;
    if (a43g_plan_build(&g, &plan)) return fail("a43g_plan_build");
    a43g_plan_sizes_t sz;
    if (a43g_plan_get_sizes(plan, &sz)) return fail("a43g_plan_get_sizes");
    std::vector<uint32_t> rowstart(size_t(sz.nRows) + 1);
    std::vector<uint16_t> colindx(size_t(sz.nnzb));
    a43g_plan_export_t ex;
    std::memset(&ex, 0, sizeof(ex));
    ex.rowstart = rowstart.data(); ex.colindx = colindx.data();
    if (a43g_plan_export(plan, &ex)) return fail("a43g_plan_export");
    bool const rows_ok = rowstart.front() == 0 && rowstart.back() == uint32_t(sz.nnzb);
    a43g_plan_destroy(plan);

    // a Hamiltonian of the same cell: zero potential, unit overlap, diagonal Hamiltonian
    int const nc = 20;                                     // numax 3
    std::vector<double> V(16*16*16, 0.0), mats(2*nc*nc, 0.0);
    for (int i = 0; i < nc; ++i) { mats[i*nc + i] = 0.1*(i + 1); mats[nc*nc + i*nc + i] = 1.0; }
    int64_t const off = 0;
    a43g_hamiltonian_t *h = nullptr;
    if (a43g_hamiltonian_create(g.ng, g.bc, g.hg, V.data(), 1, atom, mats.data(), &off, &h))
        return fail("a43g_hamiltonian_create");
    if (a43g_hamiltonian_save(h, argv[1], 0, nullptr)) return fail("a43g_hamiltonian_save");
    a43g_hamiltonian_destroy(h);
    a43g_hamiltonian_t *h2 = nullptr;
    if (a43g_hamiltonian_load(argv[1], &h2)) return fail("a43g_hamiltonian_load");
    uint32_t ng[3]; int32_t bc[3]; double hg[3]; int32_t na = 0; int64_t nmat = 0;
    if (a43g_hamiltonian_info(h2, ng, bc, hg, &na, &nmat)) return fail("a43g_hamiltonian_info");
    std::vector<double> mats2(static_cast<size_t>(nmat));
    if (a43g_hamiltonian_get(h2, nullptr, nullptr, mats2.data(), nullptr)) return fail("a43g_hamiltonian_get");
    a43g_hamiltonian_destroy(h2);
    bool mats_ok = (nmat == int64_t(mats.size()));
    // the writer keeps 16 significant digits (%.15e)
    for (size_t i = 0; mats_ok && i < mats.size(); ++i) {
        double const d = mats2[i] - mats[i], m = mats[i] < 0 ? -mats[i] : mats[i];
        mats_ok = (d <= 1e-15*m && -d <= 1e-15*m);
    }
    std::printf("{\"nnzb\": %lld, \"nRows\": %lld, \"nCols\": %lld, \"nAtoms\": %lld, \"rows_ok\": %d, "
                "\"ng\": [%u, %u, %u], \"natoms\": %d, \"mats_ok\": %d}\n",
                (long long)sz.nnzb, (long long)sz.nRows, (long long)sz.nCols, (long long)sz.nAtoms,
                rows_ok ? 1 : 0, ng[0], ng[1], ng[2], na, mats_ok ? 1 : 0);
    return (rows_ok && mats_ok && na == 1) ? 0 : 1;
}
