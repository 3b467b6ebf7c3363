// The grid Hamiltonian file (Hmt.xml / Hmt.json): reader and writer (hamiltonian_io.cpp).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace a43g {

struct Hamiltonian {
    uint32_t ng[3] = {0, 0, 0};            // grid points
    int32_t  bc[3] = {0, 0, 0};            // boundary conditions (0 isolated, 1 periodic, ...)
    double   hg[3] = {1, 1, 1};            // grid spacings (Bohr); 1 where the file gives none
    std::vector<double> Veff;              // [nz][ny][nx] local potential (Hartree)
    std::vector<double> xyzZinso;          // [natoms][8]: x, y, z (Bohr, relative to the cell centre), Z,
                                           // global id, numax, sigma, 0
    std::vector<std::vector<double>> atom_mat;   // per atom [2][nSHO][nSHO]: hamiltonian, overlap
    // returns an empty string on success, else the reason
    std::string load(char const *filename);
    std::string save(char const *filename, bool json, double const *spectrum = nullptr) const;
};

} // namespace a43g
