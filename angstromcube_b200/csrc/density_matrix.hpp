// Atomic density matrices from a Green function (density_matrix.cu).
#pragma once

#include "../../include/a43g.h"
#include "device.cuh"

namespace a43g {

struct DensityWorkspace {
    bool ready = false;                  // source-cube tables and offsets uploaded (plan geometry fixed)
    size_t nout = 0;                     // doubles of the result
    int stride = 0;                      // doubles per (image, source) table
    DeviceBuffer srcH, srcMask, out_off, out, img_index;
    DeviceBuffer apc, aac;               // image projections of G and their sums onto the atoms
};

// G: device FP64 block vector [nnzb][2][64][64]; out: host [nAtoms][nSHO][nSHO] concatenated in
// plan-atom order (synchronizes the stream)
int projection_coefficients(GreenPlan const &hp, DevicePlan &dp, DensityWorkspace &ws, double const *G,
                            double *out, cudaStream_t st);

} // namespace a43g
