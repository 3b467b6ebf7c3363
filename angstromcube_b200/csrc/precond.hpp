// Cube-diagonal preconditioner of the Green-function system (no reference counterpart: the
// reference's solver calls no preconditioner, action_t::has_preconditioner returns false).
//
// M is the local operator restricted to one 4x4x4 cube, with the cube's potential replaced by its
// mean:  M_c = Dx (+) Dy (+) Dz + (vbar_c - E) I,  D_d the finite-difference second derivative
// (times -1/(2 h_d^2)) between the cube's own four points along d.  M_c is diagonalised by the
// tensor product of the three 4x4 eigenbases Q_d of D_d, so applying M_c^-1 to a block is a
// forward transform along x, y and z, a complex scaling by 1/(lambda_x + lambda_y + lambda_z +
// vbar_c - E), and the back transform.  The solver uses it from the right: it solves
// (H - E S) M^-1 y = B and returns X = M^-1 y, so residuals and convergence are those of the
// original system.
#pragma once

#include "device.cuh"
#include "../../include/a43g.h"

namespace a43g {

struct PrecondQ { double q[3][4][4]; };    // q[d][i][k]: component i of eigenvector k of D_d
struct PrecondQf { float q[3][4][4]; };

struct BlockPreconditioner {
    PrecondQ Q{};
    PrecondQf Qf{};
    uint32_t ncells = 0, npairs = 0, nsrc_pair = 0;
    DeviceBuffer tab64, tab32;               // [npairs][ncells + 1][64][2] scaling factors
};

// the eigenbases and the scaling tables of the plan's current potential and energies (each pair
// of a batch plan with its own energy); the last cell slot serves blocks without potential.
// Returns an a43g status: A43G_ERR_ARGUMENT when a cube model is singular or its inverse not
// finite (a real energy on one of its eigenvalues), A43G_ERR_MEMORY, A43G_ERR_CUDA.
int precond_setup(GreenPlan const &hp, DevicePlan const &dp, BlockPreconditioner &pc, cudaStream_t st);

// y = M^-1 x over the blocks of the active sources (active == nullptr: every block); y may be x
template <typename T>
bool precond_apply(DevicePlan const &dp, BlockPreconditioner const &pc, T *y, T const *x, uint8_t const *active,
                   cudaStream_t st);

} // namespace a43g
