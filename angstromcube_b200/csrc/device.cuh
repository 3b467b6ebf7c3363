// Device-side plan, scratch buffers and launch interfaces shared by the CUDA sources.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include "plan.hpp"

namespace a43g {

// error state of the calling host thread (capi.cu)
void set_error(std::string const &msg);
// kernel launch counter (instrumentation, capi.cu)
void count_launch();
#define A43G_CUDA_TRY(call) do { cudaError_t e_ = (call); if (cudaSuccess != e_) { \
    ::a43g::set_error(std::string(#call) + ": " + cudaGetErrorString(e_)); return false; } } while (0)

// neighbour encoding in DevicePlan::nbr: -1 no cube (zero), >= 0 plain block index,
// <= -2 block (-e - 2) seen across a periodic boundary (multiply by the Bloch phase)
__host__ __device__ inline int32_t nbr_block(int32_t e) { return (e >= 0) ? e : (-e - 2); }

struct DeviceBuffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    bool alloc(size_t n);
    void release();
    ~DeviceBuffer() { release(); }
};

template <typename T> T *dptr(DeviceBuffer const &b) { return (T*)b.ptr; }

struct DevicePlan {
    bool uploaded = false;       // plan geometry on the device
    bool values_dirty = true;    // potential / matrices / phases need re-upload
    uint32_t nnzb = 0, nRows = 0, nCols = 0, nAtoms = 0, nAI = 0;
    uint32_t ncoeffI = 0, ncoeffA = 0;
    int lmax_max = -1;
    int FD_range[3] = {0, 0, 0};
    double prefactor[3] = {0, 0, 0};
    double phase[3][2][2] = {};
    double grid[4] = {0, 0, 0, 0};
    double E_re = 0, E_im = 0;
    bool fused_local = false;    // all directions use the 9-point stencil: fused kernel
    uint32_t max_zline = 0;      // cubes in the longest z-line
    // schedule parameters, set by the autotuner (autotune.cu) or left at these defaults
    uint32_t prj_chunk = 16;         // blocks per projection work item
    uint32_t add_blocks = 16;        // blocks per CTA of the FP32 addition
    int local_variant = 2;           // FP32: 0 rows with one-step-ahead loads, 1 plain rows, 2 pencils, 3 staged pencils
    bool local64_pencils = true;     // FP64: pencils with the planes on two threads, else the row kernel
    bool add64_unrolled = true;      // FP64 addition: z-orders unrolled, else one at a time
    bool atom_chain3 = false;        // atom matrices by the collect/multiply/broadcast kernels instead of one
    uint32_t nlists[3] = {0, 0, 0};

    DeviceBuffer veff_index;     // int32 [nnzb]
    DeviceBuffer Vcell64, Vcell32;  // [ncells][64]
    DeviceBuffer nbr;            // int32 [nnzb][6]  x-, x+, y-, y+, z-, z+
    DeviceBuffer lists_start[3], lists[3];
    DeviceBuffer colindx;        // uint16 [nnzb]
    DeviceBuffer rowindx;        // uint32 [nnzb]
    DeviceBuffer rowCubePos;     // float [nRows][4]
    DeviceBuffer prj_start, prj_col;   // [nCols][nAI+1], concatenated cols
    DeviceBuffer prj_coloff;           // uint64 [nCols]
    DeviceBuffer add_start, add_col;   // [nnzb+1], [nnz]
    DeviceBuffer sum_start, sum_col;   // [nAtoms+1], [nnz]
    DeviceBuffer img_pos, img_lmax, img_starts, img_phase;
    DeviceBuffer atom_starts, atom_lmax, atom_mat, atom_mat_off;
    DeviceBuffer grid_dev;       // double [4]: hx, hy, hz, projection radius
    DeviceBuffer subset_dev;     // uint32 [nCols] diagonal block of each source column
    DeviceBuffer slot_H, slot_mask, prj_slot, add_slot;   // projector tables per (image, row)
    DeviceBuffer slot_H32;       // float copy of slot_H for the FP32 kernels
    DeviceBuffer add_info;       // uint4 per SHOadd entry: slot, first coefficient of the image, basis size, 0
    int table_stride = 0;        // doubles per slot in slot_H
    DeviceBuffer dev_error;      // int: first error code recorded by a kernel (0: none)
    bool use_tc = true;          // FP32 projector on the tensor cores (else SIMT)
    struct ImageGroup { uint32_t count = 0; DeviceBuffer images; } img_group[8];  // images by basis size
    // SIMT projection work items by basis size: (image, source, first, last) list positions,
    // each at most kPrjChunk blocks, so that long block lists are spread over many CTAs
    // items8 adds the item's group (the items of one (image, source) pair): first item, count,
    // group index, first partial-sum slot; tickets[group] counts finished items (deterministic
    // fixed-order sum of the partials by the last one, projector_simt.cu)
    struct PrjItems { uint32_t count = 0, part_items = 0; DeviceBuffer items, items8, tickets; } prj_items[8];
    DeviceBuffer prj_part;       // partial projection sums of multi-item groups
    // batch plans (GreenPlan::replicate): npairs (energy, k-point) pairs of nsrc_pair sources each
    uint32_t npairs = 1, nsrc_pair = 0;
    size_t mat_stride = 0;       // doubles of atom matrices per pair
    DeviceBuffer pair_args32, pair_args64;   // per pair: E_re, E_im, phases [3][2][2] (float, double)
    // retirement: sources whose columns have all finished are skipped by every kernel of the
    // action and of the solver while retire is set (uint8 per source, 1 = active)
    bool retire = false;
    DeviceBuffer src_active;
    // the blocks of every source in order (the solver's fixed-order column reductions)
    DeviceBuffer src_start, src_blocks;      // uint32 [nCols + 1], uint32 [nnzb]
    uint32_t max_src_blocks = 0;
    // scratch of the dyadic part (allocated once per plan, never per call)
    DeviceBuffer apc;            // real_t [ncoeffI*nCols][2][64] image projection coefficients
    DeviceBuffer aac, cadd;      // double [ncoeffA*nCols][2][64]
    DeviceBuffer cad;            // real_t [ncoeffI*nCols][2][64] image addition coefficients
    size_t apc_elem_bytes = 0;   // 4 or 8: precision the apc/cad scratch is sized for
};

bool upload_plan(GreenPlan const &hp, DevicePlan &dp);
// kernel attributes (dynamic shared memory above 48 KB) of the current device
bool prepare_simt_kernels();
bool prepare_local_kernels();
bool prepare_tc_kernels();
// kernel launch counter: n launches at once (replays of a captured graph)
void count_launches(uint64_t n);
uint64_t launches_so_far();
bool upload_values(GreenPlan const &hp, DevicePlan &dp);
// projection work items (image, source, up to dp.prj_chunk consecutive blocks of its list)
bool build_prj_items(GreenPlan const &hp, DevicePlan &dp);
// chooses the schedule parameters of the action for this plan by timing them (autotune.cu)
template <typename T>
bool autotune(GreenPlan const &hp, DevicePlan &dp, cudaStream_t st, std::string &report);
bool ensure_dyadic_scratch(DevicePlan &dp, size_t elem_bytes);
// partial-sum buffer of the deterministic SIMT projection for reals of elem_bytes
bool ensure_prj_part(DevicePlan &dp, size_t elem_bytes);

// the action y = (H - E S) x on real_t = double or float
template <typename T>
bool launch_action(DevicePlan &dp, T *y, T const *x, uint16_t const *colIndex, cudaStream_t s);

// parts of the action (tests, VJP and benchmarks use them separately)
template <typename T>
bool launch_local(DevicePlan &dp, T *y, T const *x, cudaStream_t s);          // potential + kinetic
template <typename T>
bool launch_dyadic(DevicePlan &dp, T *y, T const *x, uint16_t const *colIndex, cudaStream_t s);

double action_flops(GreenPlan const &hp, int real_bytes);

// the action with the dyadic coefficients in caller-given scratch instead of the plan's
// buffers: apc, cad hold ncoeffI*nCols*128 reals of the action's precision, aac, cadd
// ncoeffA*nCols*128 doubles (apc is zeroed by the call; the others are overwritten)
struct DyadicScratch { void *apc, *cad; double *aac, *cadd; };
template <typename T>
bool launch_action_scratch(DevicePlan &dp, T *y, T const *x, uint16_t const *colIndex, cudaStream_t st,
                           DyadicScratch const &sc);

// FP64 pieces of the dyadic part on caller-given buffers (vector-Jacobian products):
// apc = P x with the given projector tables (zeroed first); aac = sum over images of
// img_phase * apc; out = M in (atom matrices of the plan)
bool launch_project_with(DevicePlan &dp, double *apc, double const *x, double const *table, cudaStream_t st);
bool launch_collect_with(DevicePlan &dp, double *aac, double const *apc, double const *img_phase, cudaStream_t st);
bool launch_mul_with(DevicePlan &dp, double *out, double const *in, cudaStream_t st);

// tensor-core (tcgen05, 3xTF32) projection and addition of the FP32 action (projector_tc.cu)
bool tc_projector_supported(DevicePlan const &dp);
bool launch_project_tc(DevicePlan &dp, float const *x, cudaStream_t st);
bool launch_add_tc(DevicePlan &dp, float *y, uint16_t const *colIndex, cudaStream_t st);

// sum-factorized projection and addition on the CUDA cores (projector_simt.cu, FP32 and FP64);
// both stage blocks with 16-byte copies and need 16-byte aligned x and y
bool simt_projector_supported(DevicePlan const &dp, void const *x, void const *y, size_t real_bytes);
template <typename T> bool launch_project_simt(DevicePlan &dp, T const *x, cudaStream_t st);
template <typename T> bool launch_add_simt(DevicePlan &dp, T *y, uint16_t const *colIndex, cudaStream_t st);

} // namespace a43g
