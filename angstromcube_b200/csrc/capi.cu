// extern "C" entry points declared in include/a43g.h.
#include "../../include/a43g.h"
#include "device.cuh"
#include "solver.hpp"
#include "vjp.hpp"
#include "noalloc.hpp"
#include "hamiltonian_io.hpp"
#include "density_matrix.hpp"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <new>

struct a43g_plan {
    a43g::GreenPlan host;
    a43g::DevicePlan dev;
    a43g::SolverWorkspace solver;
    a43g::BatchCache batch;          // batch plan and vectors of a43g_solve_batched
    a43g::DensityWorkspace density;  // tables and scratch of a43g_projection_coefficients
    a43g::VjpWorkspace vjpws;
    bool energy_set = false;
    bool matrices_set = false;
    int device = -1;
    std::mutex mtx;                  // calls on one plan are serialised; distinct plans are independent
};

namespace a43g {
namespace {
thread_local std::string g_error;
std::atomic<uint64_t> g_launches{0};
}
void set_error(std::string const &msg) { g_error = msg; }
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void count_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
uint64_t launches_so_far() { return g_launches.load(std::memory_order_relaxed); }
} // namespace a43g

using a43g::set_error;

namespace {

int fail(int code, std::string const &msg) { set_error(msg); return code; }

int ensure_device(a43g_plan_t *p) {
    int dev = 0;
    if (cudaSuccess != cudaGetDevice(&dev)) return fail(A43G_ERR_CUDA, "no CUDA device available");
    if (p->device >= 0 && p->device != dev) return fail(A43G_ERR_STATE, "plan was uploaded to another device");
    if (!p->dev.uploaded) {
        if (!a43g::upload_plan(p->host, p->dev)) return A43G_ERR_CUDA;
        p->device = dev;
    } else if (p->dev.values_dirty) {
        if (!a43g::upload_values(p->host, p->dev)) return A43G_ERR_CUDA;
    }
    return A43G_OK;
}

} // namespace

extern "C" {

const char *a43g_last_error(void) { return a43g::g_error.c_str(); }

const char *a43g_version(void) { return "a43g 0.1 (sm_100a)"; }

namespace {

int build_plan(const a43g_geometry_t *g, a43g_plan_t **plan, a43g::ImageRowsFn image_rows) {
    if (!g || !plan) return fail(A43G_ERR_ARGUMENT, "null argument");
    if (g->natoms < 0 || (g->natoms > 0 && !g->xyzZinso)) return fail(A43G_ERR_ARGUMENT, "atoms missing");
    auto *p = new (std::nothrow) a43g_plan();
    if (!p) return fail(A43G_ERR_MEMORY, "host allocation failed");
    a43g::Geometry geo;
    for (int d = 0; d < 3; ++d) {
        geo.ng[d] = g->ng[d]; geo.bc[d] = int8_t(g->bc[d]); geo.hg[d] = g->hg[d]; geo.sources[d] = g->sources[d];
    }
    geo.r_trunc = g->r_trunc; geo.nFD = g->nFD; geo.proj_radius = g->proj_radius;
    geo.xyzZinso.assign(g->xyzZinso, g->xyzZinso + 8*size_t(g->natoms));
    std::string err;
    try { err = p->host.build(geo, image_rows); } catch (std::bad_alloc const &) { err = "host memory exhausted"; }
    if (!err.empty()) {
        delete p;
        bool const device = 0 == err.rfind("device plan construction", 0);
        return fail(device ? A43G_ERR_CUDA : A43G_ERR_ARGUMENT, err);
    }
    *plan = p;
    return A43G_OK;
}

} // namespace

int a43g_plan_build(const a43g_geometry_t *g, a43g_plan_t **plan) { return build_plan(g, plan, nullptr); }

int a43g_plan_build_device(const a43g_geometry_t *g, a43g_plan_t **plan) {
    return build_plan(g, plan, a43g::image_rows_on_device);
}

int a43g_plan_destroy(a43g_plan_t *plan) {
    if (!plan) return A43G_OK;
    if (plan->device >= 0) cudaSetDevice(plan->device);
    delete plan;
    return A43G_OK;
}

int a43g_plan_get_sizes(const a43g_plan_t *plan, a43g_plan_sizes_t *s) {
    if (!plan || !s) return fail(A43G_ERR_ARGUMENT, "null argument");
    auto const &h = plan->host;
    s->nnzb = int64_t(h.nnzb()); s->nRows = h.nRows; s->nCols = h.nCols;
    s->nAtoms = h.nAtoms; s->nAtomImages = h.nAtomImages;
    s->ncoeff_images = int64_t(h.ncoeff_images()); s->ncoeffs = int64_t(h.ncoeff_atoms());
    for (int d = 0; d < 3; ++d) {
        s->nlists[d] = h.kinetic[d].nlists(); s->lists_nnz[d] = int64_t(h.kinetic[d].entry.size());
        s->FD_range[d] = h.kinetic[d].FD_range;
    }
    s->SHOadd_nnz = h.SHOadd.nnz();
    int64_t n = 0; for (auto const &c : h.SHOprj) n += c.nnz();
    s->SHOprj_nnz = n;
    s->SHOsum_nnz = h.SHOsum.nnz();
    s->ncells = int64_t(h.ncells());
    return A43G_OK;
}

int a43g_plan_export(const a43g_plan_t *plan, const a43g_plan_export_t *e) {
    if (!plan || !e) return fail(A43G_ERR_ARGUMENT, "null argument");
    auto const &h = plan->host;
    auto cp = [](void *dst, void const *src, size_t bytes) { if (dst && bytes) std::memcpy(dst, src, bytes); };
    size_t const nnzb = h.nnzb();
    cp(e->rowstart, h.rowstart.data(), h.rowstart.size()*4);
    cp(e->colindx, h.colindx.data(), nnzb*2);
    cp(e->rowindx, h.rowindx.data(), nnzb*4);
    cp(e->veff_index, h.veff_index.data(), nnzb*4);
    cp(e->subset, h.subset.data(), h.subset.size()*4);
    cp(e->rowCubePos, h.rowCubePos.data(), h.rowCubePos.size()*4);
    cp(e->colCubePos, h.colCubePos.data(), h.colCubePos.size()*4);
    cp(e->target_minus_source, h.target_minus_source.data(), h.target_minus_source.size()*2);
    cp(e->grid_spacing_trunc, h.h_trunc, 24);
    for (int d = 0; d < 3; ++d) {
        if (e->kinetic_prefactor) e->kinetic_prefactor[d] = h.kinetic[d].prefactor;
        cp(e->lists_start[d], h.kinetic[d].start.data(), h.kinetic[d].start.size()*4);
        cp(e->lists[d], h.kinetic[d].entry.data(), h.kinetic[d].entry.size()*4);
    }
    cp(e->AtomStarts, h.AtomStarts.data(), h.AtomStarts.size()*4);
    cp(e->AtomLmax, h.AtomLmax.data(), h.AtomLmax.size());
    cp(e->AtomSigma, h.AtomSigma.data(), h.AtomSigma.size()*8);
    cp(e->global_atom_ids, h.global_atom_ids.data(), h.global_atom_ids.size()*8);
    cp(e->AtomImageIndex, h.AtomImageIndex.data(), h.AtomImageIndex.size()*4);
    cp(e->AtomImageStarts, h.AtomImageStarts.data(), h.AtomImageStarts.size()*4);
    cp(e->AtomImagePos, h.AtomImagePos.data(), h.AtomImagePos.size()*8);
    cp(e->AtomImageLmax, h.AtomImageLmax.data(), h.AtomImageLmax.size());
    cp(e->AtomImageShift, h.AtomImageShift.data(), h.AtomImageShift.size());
    cp(e->AtomImagePhase, h.AtomImagePhase.data(), h.AtomImagePhase.size()*8);
    cp(e->grid_spacing_dyadic, h.grid_spacing_dyadic, 32);
    cp(e->SHOadd_start, h.SHOadd.start.data(), h.SHOadd.start.size()*4);
    cp(e->SHOadd_col, h.SHOadd.col.data(), h.SHOadd.col.size()*4);
    if (e->SHOprj_start || e->SHOprj_col) {
        size_t os = 0, oc = 0;
        for (auto const &c : h.SHOprj) {
            if (e->SHOprj_start) {
                if (c.start.empty()) std::memset(e->SHOprj_start + os, 0, (h.nAtomImages + 1)*4);
                else std::memcpy(e->SHOprj_start + os, c.start.data(), c.start.size()*4);
            }
            os += h.nAtomImages + 1;
            if (e->SHOprj_col) cp(e->SHOprj_col + oc, c.col.data(), c.col.size()*4);
            oc += c.col.size();
        }
    }
    cp(e->SHOsum_start, h.SHOsum.start.data(), h.SHOsum.start.size()*4);
    cp(e->SHOsum_col, h.SHOsum.col.data(), h.SHOsum.col.size()*4);
    cp(e->AtomMatrices, h.AtomMatrices.data(), h.AtomMatrices.size()*8);
    cp(e->phase, h.phase, 12*8);
    return A43G_OK;
}

int a43g_plan_set_potential(a43g_plan_t *plan, const double *V, int layout) {
    if (!plan || !V) return fail(A43G_ERR_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(plan->mtx);
    if (0 == layout) plan->host.set_potential_grid(V);
    else if (1 == layout) plan->host.set_potential_cells(V);
    else return fail(A43G_ERR_ARGUMENT, "layout must be 0 (grid) or 1 (cell cubes)");
    plan->dev.values_dirty = true;
    return A43G_OK;
}

int a43g_plan_set_atom_matrices(a43g_plan_t *plan, const double *mats, const int64_t *offsets, int64_t natoms) {
    if (!plan || (!mats && natoms > 0) || (!offsets && natoms > 0)) return fail(A43G_ERR_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(plan->mtx);
    auto const err = plan->host.set_atom_matrices(mats, offsets, natoms);
    if (!err.empty()) return fail(A43G_ERR_ARGUMENT, err);
    plan->matrices_set = true;
    plan->dev.values_dirty = true;
    return A43G_OK;
}

int a43g_plan_set_energy(a43g_plan_t *plan, double Er, double Ei, double dVol) {
    if (!plan) return fail(A43G_ERR_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(plan->mtx);
    plan->host.set_energy(Er, Ei, dVol);
    plan->energy_set = true;
    plan->dev.values_dirty = true;
    return A43G_OK;
}

int a43g_plan_set_kpoint(a43g_plan_t *plan, const double k[3]) {
    if (!plan || !k) return fail(A43G_ERR_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(plan->mtx);
    auto const err = plan->host.set_kpoint(k);
    if (!err.empty()) return fail(A43G_ERR_ARGUMENT, err);
    plan->dev.values_dirty = true;
    return A43G_OK;
}

int a43g_plan_upload(a43g_plan_t *plan) {
    if (!plan) return fail(A43G_ERR_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(plan->mtx);
    return ensure_device(plan);
}

int a43g_action_multiply(a43g_plan_t *plan, void *y, const void *x, const uint16_t *colIndex,
                         uint32_t nnzb, uint32_t nCols, unsigned /*l2nX*/, void *stream, int dtype,
                         double *flops) {
    if (!plan || (!y && nnzb) || (!x && nnzb) || (!colIndex && nnzb)) return fail(A43G_ERR_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(plan->mtx);
    if (nnzb != plan->host.nnzb()) return fail(A43G_ERR_ARGUMENT, "nnzb does not match the plan");
    if (nCols != plan->host.nCols) return fail(A43G_ERR_ARGUMENT, "nCols does not match the plan");
    if (!plan->energy_set) return fail(A43G_ERR_STATE, "energy parameter not set (a43g_plan_set_energy)");
    if (y == x) return fail(A43G_ERR_ARGUMENT, "y and x must not alias");
    int const rc = ensure_device(plan);
    if (rc) return rc;
    auto const st = (cudaStream_t)stream;
    bool ok;
    if (A43G_F64 == dtype) ok = a43g::launch_action<double>(plan->dev, (double*)y, (double const*)x, colIndex, st);
    else if (A43G_F32 == dtype) ok = a43g::launch_action<float>(plan->dev, (float*)y, (float const*)x, colIndex, st);
    else return fail(A43G_ERR_ARGUMENT, "dtype must be A43G_F64 or A43G_F32");
    if (!ok) return A43G_ERR_CUDA;
    if (flops) *flops = a43g::action_flops(plan->host, (A43G_F64 == dtype) ? 8 : 4);
    return A43G_OK;
}

int a43g_action_multiply_noalloc(a43g_plan_t *plan, void *y, const void *x, const uint16_t *colIndex,
                                 uint32_t nnzb, uint32_t nCols, void *stream, int dtype, double *flops) {
    if (!plan || (!y && nnzb) || (!x && nnzb) || (!colIndex && nnzb)) return fail(A43G_ERR_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(plan->mtx);
    if (nnzb != plan->host.nnzb()) return fail(A43G_ERR_ARGUMENT, "nnzb does not match the plan");
    if (nCols != plan->host.nCols) return fail(A43G_ERR_ARGUMENT, "nCols does not match the plan");
    if (!plan->energy_set) return fail(A43G_ERR_STATE, "energy parameter not set (a43g_plan_set_energy)");
    if (y == x) return fail(A43G_ERR_ARGUMENT, "y and x must not alias");
    if (A43G_F64 != dtype && A43G_F32 != dtype) return fail(A43G_ERR_ARGUMENT, "dtype must be A43G_F64 or A43G_F32");
    // this entry point never uploads (uploading allocates): the plan must be current on this device
    int dev = -1;
    if (cudaSuccess != cudaGetDevice(&dev)) return fail(A43G_ERR_CUDA, "no CUDA device available");
    if (!plan->dev.uploaded || plan->device != dev || plan->dev.values_dirty)
        return fail(A43G_ERR_STATE, "the plan is not current on this device: call a43g_plan_upload after the last "
                                    "change of potential, matrices, energy or k-point");
    size_t const need = a43g::noalloc_required(plan->dev, (A43G_F64 == dtype) ? 8 : 4);
    if (need > a43g::noalloc_capacity())
        return fail(A43G_ERR_UNSUPPORTED, "the projector coefficients of this plan need " + std::to_string(need) +
                    " bytes of scratch, more than the " + std::to_string(a43g::noalloc_capacity()) +
                    " bytes of the allocation-free entry point; use a43g_action_multiply");
    auto const st = (cudaStream_t)stream;
    bool const ok = (A43G_F64 == dtype)
        ? a43g::action_noalloc<double>(plan->dev, (double*)y, (double const*)x, colIndex, st)
        : a43g::action_noalloc<float>(plan->dev, (float*)y, (float const*)x, colIndex, st);
    if (!ok) return A43G_ERR_CUDA;
    if (flops) *flops = a43g::action_flops(plan->host, (A43G_F64 == dtype) ? 8 : 4);
    return A43G_OK;
}

int a43g_plan_autotune(a43g_plan_t *plan, int dtype, void *stream, char *report, size_t report_size) {
    if (!plan) return fail(A43G_ERR_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(plan->mtx);
    if (!plan->energy_set) return fail(A43G_ERR_STATE, "energy parameter not set (a43g_plan_set_energy)");
    int const rc = ensure_device(plan);
    if (rc) return rc;
    std::string text;
    bool ok;
    if (A43G_F64 == dtype) ok = a43g::autotune<double>(plan->host, plan->dev, (cudaStream_t)stream, text);
    else if (A43G_F32 == dtype) ok = a43g::autotune<float>(plan->host, plan->dev, (cudaStream_t)stream, text);
    else return fail(A43G_ERR_ARGUMENT, "dtype must be A43G_F64 or A43G_F32");
    if (report && report_size) {
        size_t const m = std::min(report_size - 1, text.size());
        std::memcpy(report, text.data(), m);
        report[m] = 0;
    }
    return ok ? A43G_OK : A43G_ERR_CUDA;
}

int a43g_vjp(a43g_plan_t *plan, const void *L, const void *G, double *dV, double *dM, double *dR, void *stream) {
    if (!plan || !L || !G) return fail(A43G_ERR_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(plan->mtx);
    if (!plan->energy_set) return fail(A43G_ERR_STATE, "energy parameter not set (a43g_plan_set_energy)");
    int const rc = ensure_device(plan);
    if (rc) return rc;
    return a43g::vjp(plan->host, plan->dev, plan->vjpws, (double const*)L, (double const*)G, dV, dM, dR,
                     (cudaStream_t)stream);
}

int a43g_action_part(a43g_plan_t *plan, int part, void *y, const void *x, void *stream, int dtype) {
    if (!plan || !y || !x) return fail(A43G_ERR_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(plan->mtx);
    if (!plan->energy_set) return fail(A43G_ERR_STATE, "energy parameter not set (a43g_plan_set_energy)");
    int const rc = ensure_device(plan);
    if (rc) return rc;
    auto const st = (cudaStream_t)stream;
    auto const *ci = a43g::dptr<uint16_t>(plan->dev.colindx);
    bool ok;
    if (0 == part && A43G_F64 == dtype) ok = a43g::launch_local<double>(plan->dev, (double*)y, (double const*)x, st);
    else if (0 == part && A43G_F32 == dtype) ok = a43g::launch_local<float>(plan->dev, (float*)y, (float const*)x, st);
    else if (1 == part && A43G_F64 == dtype) ok = a43g::launch_dyadic<double>(plan->dev, (double*)y, (double const*)x, ci, st);
    else if (1 == part && A43G_F32 == dtype) ok = a43g::launch_dyadic<float>(plan->dev, (float*)y, (float const*)x, ci, st);
    else return fail(A43G_ERR_ARGUMENT, "part must be 0 or 1, dtype A43G_F64 or A43G_F32");
    return ok ? A43G_OK : A43G_ERR_CUDA;
}

uint64_t a43g_kernel_launches(void) { return a43g::g_launches.load(); }

int a43g_plan_device_status(a43g_plan_t *plan) {
    if (!plan) return fail(A43G_ERR_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(plan->mtx);
    if (cudaSuccess != cudaDeviceSynchronize()) return fail(A43G_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
    if (!plan->dev.dev_error.ptr) return A43G_OK;
    int32_t code = 0;
    if (cudaSuccess != cudaMemcpy(&code, plan->dev.dev_error.ptr, 4, cudaMemcpyDeviceToHost)) return fail(A43G_ERR_CUDA, "copy of the error flag");
    if (0 == code) return A43G_OK;
    cudaMemset(plan->dev.dev_error.ptr, 0, 4);
    return fail(A43G_ERR_CUDA, std::string("a kernel recorded error ") + std::to_string(code) +
                (code <= 2 ? " (tensor-core projector wait timed out)" : ""));
}

int a43g_solve(a43g_plan_t *plan, const a43g_solve_options_t *opts, void *X, double *rho,
               a43g_solve_stats_t *stats, void *stream) {
    if (!plan || !opts) return fail(A43G_ERR_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(plan->mtx);
    if (!plan->energy_set) return fail(A43G_ERR_STATE, "energy parameter not set (a43g_plan_set_energy)");
    int const rc = ensure_device(plan);
    if (rc) return rc;
    a43g_solve_stats_t local{};
    int const r = a43g::solve(plan->host, plan->dev, plan->solver, *opts, X, rho, stats ? stats : &local,
                              (cudaStream_t)stream);
    return r;
}

int a43g_solve_traced(a43g_plan_t *plan, const a43g_solve_options_t *opts, void *X, double *rho,
                      a43g_solve_stats_t *stats, void *stream, const void *X_reference, int32_t every,
                      double *trace, int32_t capacity, int32_t *count) {
    if (!plan || !opts || !X_reference || (capacity > 0 && !trace)) return fail(A43G_ERR_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(plan->mtx);
    if (!plan->energy_set) return fail(A43G_ERR_STATE, "energy parameter not set (a43g_plan_set_energy)");
    int const rc = ensure_device(plan);
    if (rc) return rc;
    a43g_solve_stats_t local{};
    a43g::SolveTrace tr;
    tr.Xref = static_cast<double const*>(X_reference);
    tr.every = std::max<int32_t>(1, every);
    int const r = a43g::solve(plan->host, plan->dev, plan->solver, *opts, X, rho, stats ? stats : &local,
                              (cudaStream_t)stream, nullptr, &tr);
    int32_t const nrow = int32_t(tr.rows.size()/3);
    int32_t const keep = std::min(nrow, std::max<int32_t>(0, capacity));
    if (keep > 0) std::copy(tr.rows.begin(), tr.rows.begin() + 3*size_t(keep), trace);
    if (count) *count = nrow;
    return r;
}

int a43g_solve_batched(a43g_plan_t *plan, const a43g_solve_options_t *opts, int32_t n,
                       const double *energies, const double *kpoints, double dVol,
                       double *rho, a43g_solve_stats_t *stats, void *stream) {
    if (!plan || !opts || n < 0 || (n > 0 && (!energies || !kpoints || !stats)))
        return fail(A43G_ERR_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(plan->mtx);
    if (!plan->matrices_set && plan->host.nAtoms > 0) return fail(A43G_ERR_STATE, "atom matrices not set");
    int const rc = ensure_device(plan);
    if (rc) return rc;
    return a43g::solve_batched(plan->host, plan->dev, plan->batch, *opts, n, energies, kpoints, dVol,
                               rho, stats, (cudaStream_t)stream);
}

int a43g_projection_coefficients(a43g_plan_t *plan, const void *G, double *out, void *stream) {
    if (!plan || !G || !out) return fail(A43G_ERR_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(plan->mtx);
    if (!plan->energy_set) return fail(A43G_ERR_STATE, "energy parameter not set (a43g_plan_set_energy)");
    int const rc = ensure_device(plan);
    if (rc) return rc;
    return a43g::projection_coefficients(plan->host, plan->dev, plan->density, (double const*)G, out,
                                         (cudaStream_t)stream);
}

struct a43g_hamiltonian { a43g::Hamiltonian h; };

int a43g_hamiltonian_load(const char *filename, a43g_hamiltonian_t **h) {
    if (!filename || !h) return fail(A43G_ERR_ARGUMENT, "null argument");
    auto *p = new (std::nothrow) a43g_hamiltonian();
    if (!p) return fail(A43G_ERR_MEMORY, "host allocation failed");
    std::string err;
    try { err = p->h.load(filename); } catch (std::bad_alloc const &) { err = "host memory exhausted"; }
    if (!err.empty()) { delete p; return fail(A43G_ERR_ARGUMENT, err); }
    *h = p;
    return A43G_OK;
}

int a43g_hamiltonian_info(const a43g_hamiltonian_t *h, uint32_t ng[3], int32_t bc[3], double hg[3],
                          int32_t *natoms, int64_t *nmat) {
    if (!h) return fail(A43G_ERR_ARGUMENT, "null argument");
    for (int d = 0; d < 3; ++d) {
        if (ng) ng[d] = h->h.ng[d];
        if (bc) bc[d] = h->h.bc[d];
        if (hg) hg[d] = h->h.hg[d];
    }
    if (natoms) *natoms = int32_t(h->h.atom_mat.size());
    if (nmat) { int64_t n = 0; for (auto const &m : h->h.atom_mat) n += int64_t(m.size()); *nmat = n; }
    return A43G_OK;
}

int a43g_hamiltonian_get(const a43g_hamiltonian_t *h, double *Veff, double *xyzZinso, double *mats, int64_t *offsets) {
    if (!h) return fail(A43G_ERR_ARGUMENT, "null argument");
    if (Veff) std::memcpy(Veff, h->h.Veff.data(), h->h.Veff.size()*sizeof(double));
    if (xyzZinso) std::memcpy(xyzZinso, h->h.xyzZinso.data(), h->h.xyzZinso.size()*sizeof(double));
    int64_t o = 0;
    for (size_t a = 0; a < h->h.atom_mat.size(); ++a) {
        if (offsets) offsets[a] = o;
        if (mats) std::memcpy(mats + o, h->h.atom_mat[a].data(), h->h.atom_mat[a].size()*sizeof(double));
        o += int64_t(h->h.atom_mat[a].size());
    }
    return A43G_OK;
}

int a43g_hamiltonian_create(const uint32_t ng[3], const int32_t bc[3], const double hg[3], const double *Veff,
                            int32_t natoms, const double *xyzZinso, const double *mats, const int64_t *offsets,
                            a43g_hamiltonian_t **h) {
    if (!ng || !bc || !hg || !Veff || !h || natoms < 0 || (natoms > 0 && (!xyzZinso || !mats || !offsets)))
        return fail(A43G_ERR_ARGUMENT, "null argument");
    auto *p = new (std::nothrow) a43g_hamiltonian();
    if (!p) return fail(A43G_ERR_MEMORY, "host allocation failed");
    for (int d = 0; d < 3; ++d) { p->h.ng[d] = ng[d]; p->h.bc[d] = bc[d]; p->h.hg[d] = hg[d]; }
    p->h.Veff.assign(Veff, Veff + size_t(ng[0])*ng[1]*ng[2]);
    p->h.xyzZinso.assign(xyzZinso, xyzZinso + 8*size_t(natoms));
    for (int32_t a = 0; a < natoms; ++a) {
        int const numax = int(xyzZinso[8*a + 5]);
        if (numax < 0 || numax > 15) { delete p; return fail(A43G_ERR_ARGUMENT, "numax out of range"); }
        int const nc = ((1 + numax)*(2 + numax)*(3 + numax))/6;
        p->h.atom_mat.emplace_back(mats + offsets[a], mats + offsets[a] + 2*size_t(nc)*nc);
    }
    *h = p;
    return A43G_OK;
}

int a43g_hamiltonian_save(const a43g_hamiltonian_t *h, const char *filename, int format, const double *spectrum) {
    if (!h || !filename) return fail(A43G_ERR_ARGUMENT, "null argument");
    if (0 != format && 1 != format) return fail(A43G_ERR_ARGUMENT, "format must be 0 (XML) or 1 (JSON)");
    auto const err = h->h.save(filename, 1 == format, spectrum);
    return err.empty() ? A43G_OK : fail(A43G_ERR_ARGUMENT, err);
}

int a43g_hamiltonian_destroy(a43g_hamiltonian_t *h) {
    delete h;
    return A43G_OK;
}

} // extern "C"
