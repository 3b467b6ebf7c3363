// Vector-Jacobian products of the action (vjp.cu).
#pragma once

#include "../../include/a43g.h"
#include "device.cuh"

namespace a43g {

struct VjpWorkspace {
    DeviceBuffer dV, dM, dR;                  // device results
    DeviceBuffer apc, lA, gA;                 // image projections, collected projections of L and G
    DeviceBuffer Mg, dl, dg, Mdg;             // position derivatives
    DeviceBuffer phase_conj;                  // conjugated image phases
    DeviceBuffer slot_Hd[3];                  // projector tables differentiated along x, y, z
    bool tables_ready = false;                // slot_Hd uploaded (the plan geometry is fixed)
};

// L, G: device FP64 block vectors [nnzb][2][64][64]; dV, dM, dR: host outputs or null
// (layouts in include/a43g.h, a43g_vjp); synchronizes the stream
int vjp(GreenPlan const &hp, DevicePlan &dp, VjpWorkspace &ws, double const *L, double const *G,
        double *dV, double *dM, double *dR, cudaStream_t st);

} // namespace a43g
