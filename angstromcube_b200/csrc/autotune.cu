// Autotuner of the action's schedule for one plan on the current device.
//
// The kernels have a few schedule parameters whose best value depends on the plan (how many
// blocks, how many atom images per block, how long the z-lines are) and on the GPU:
//   * prj_chunk   : blocks of one (image, source) list per projection CTA (the cubes-per-CTA
//                   schedule of the projection: longer chunks amortize the pipeline start and
//                   the coefficient atomics, shorter ones balance the load)   {8, 16, 32}
//   * add_blocks  : consecutive blocks per CTA of the FP32 addition        {8, 16, 32}
//   * local_variant: FP32 local kernel on rows with one-step-ahead loads, on plain rows, on
//                   y-pencils, or on y-pencils with staged neighbour cubes     {0, 1, 2, 3}
//   * use_tc      : FP32 projector on the tensor cores (3xTF32) or on the CUDA cores
//   * local64_pencils: FP64 local kernel on pencils (planes on two threads) or on rows
// Each parameter is tuned in turn (coordinate descent), every candidate timed with CUDA events
// on the caller's stream: two untimed applications, then the mean of three.  Scratch vectors
// for x and y are allocated for the duration of the call.
#include "device.cuh"

#include <cstdio>
#include <string>
#include <vector>

namespace a43g {

namespace {

template <typename T>
bool time_part(DevicePlan &dp, int part, T *y, T const *x, uint16_t const *ci, cudaStream_t st, float &ms) {
    cudaEvent_t e0, e1;
    A43G_CUDA_TRY(cudaEventCreate(&e0));
    A43G_CUDA_TRY(cudaEventCreate(&e1));
    auto run = [&]() {
        return (0 == part) ? launch_local<T>(dp, y, x, st) : launch_dyadic<T>(dp, y, x, ci, st);
    };
    bool ok = run() && run();
    if (ok) {
        cudaEventRecord(e0, st);
        for (int r = 0; r < 3 && ok; ++r) ok = run();
        cudaEventRecord(e1, st);
        ok = ok && cudaSuccess == cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        ms /= 3;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ok;
}

} // namespace

template <typename T>
bool autotune(GreenPlan const &hp, DevicePlan &dp, cudaStream_t st, std::string &report) {
    size_t const n = size_t(dp.nnzb)*8192;
    if (0 == n) return true;
    DeviceBuffer bx, by;
    if (!bx.alloc(n*sizeof(T)) || !by.alloc(n*sizeof(T))) return false;
    A43G_CUDA_TRY(cudaMemsetAsync(bx.ptr, 0x3c, n*sizeof(T), st));   // finite values of moderate size
    T *y = dptr<T>(by);
    T const *x = dptr<T>(bx);
    uint16_t const *ci = dptr<uint16_t>(dp.colindx);
    char line[160];
    float ms = 0;
    if (dp.nAI > 0 && dp.nCols > 0) {
        uint32_t best = dp.prj_chunk; float tbest = 1e30f;
        for (uint32_t c : {8u, 16u, 32u}) {
            dp.prj_chunk = c;
            if (!build_prj_items(hp, dp) || !time_part<T>(dp, 1, y, x, ci, st, ms)) return false;
            std::snprintf(line, sizeof(line), "projector chunk %2u blocks: %.3f ms\n", c, ms); report += line;
            if (ms < tbest) { tbest = ms; best = c; }
        }
        dp.prj_chunk = best;
        if (!build_prj_items(hp, dp)) return false;
        if (sizeof(T) == 4) {
            uint32_t bestb = dp.add_blocks; tbest = 1e30f;
            for (uint32_t c : {8u, 16u, 32u}) {
                dp.add_blocks = c;
                if (!time_part<T>(dp, 1, y, x, ci, st, ms)) return false;
                std::snprintf(line, sizeof(line), "addition %2u blocks per CTA: %.3f ms\n", c, ms); report += line;
                if (ms < tbest) { tbest = ms; bestb = c; }
            }
            dp.add_blocks = bestb;
            if (tc_projector_supported(dp)) {
                bool const before = dp.use_tc;
                float t[2] = {0, 0};
                for (int tc = 0; tc < 2; ++tc) {
                    dp.use_tc = (1 == tc);
                    if (!time_part<T>(dp, 1, y, x, ci, st, t[tc])) { dp.use_tc = before; return false; }
                    std::snprintf(line, sizeof(line), "projector on the %s: %.3f ms\n", tc ? "tensor cores" : "CUDA cores", t[tc]);
                    report += line;
                }
                dp.use_tc = t[1] < t[0];
                if (dp.use_tc) {   // a tensor-core run that recorded a wait timeout is not usable
                    int flag = 0;
                    A43G_CUDA_TRY(cudaMemcpyAsync(&flag, dp.dev_error.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
                    A43G_CUDA_TRY(cudaStreamSynchronize(st));
                    if (flag) dp.use_tc = false;
                }
            }
        }
    }
    char const *const local_name[4] = {"rows with loads ahead", "plain rows", "pencils", "staged pencils"};
    if (sizeof(T) == 4 && dp.fused_local) {
        float t[4] = {0, 0, 0, 0};
        int best = 0;
        for (int v = 0; v < 4; ++v) {
            dp.local_variant = v;
            if (!time_part<T>(dp, 0, y, x, ci, st, t[v])) return false;
            std::snprintf(line, sizeof(line), "local kernel, %s: %.3f ms\n", local_name[v], t[v]);
            report += line;
            if (t[v] < t[best]) best = v;
        }
        dp.local_variant = best;
    }
    if (sizeof(T) == 8 && dp.fused_local) {
        float t[2] = {0, 0};
        for (int v = 0; v < 2; ++v) {
            dp.local64_pencils = (1 == v);
            if (!time_part<T>(dp, 0, y, x, ci, st, t[v])) return false;
            std::snprintf(line, sizeof(line), "FP64 local kernel, %s: %.3f ms\n", v ? "pencils" : "rows", t[v]);
            report += line;
        }
        dp.local64_pencils = t[1] <= t[0];
    }
    if (sizeof(T) == 8 && dp.nAI > 0 && dp.nCols > 0) {
        float t[2] = {0, 0};
        for (int v = 0; v < 2; ++v) {
            dp.add64_unrolled = (1 == v);
            if (!time_part<T>(dp, 1, y, x, ci, st, t[v])) return false;
            std::snprintf(line, sizeof(line), "FP64 projector, addition %s: %.3f ms\n", v ? "unrolled" : "rolled", t[v]);
            report += line;
        }
        dp.add64_unrolled = t[1] <= t[0];
    }
    std::snprintf(line, sizeof(line), "chosen: projector chunk %u, addition %u blocks per CTA, local %s, %s projector\n",
                  dp.prj_chunk, dp.add_blocks, local_name[dp.local_variant],
                  dp.use_tc ? "tensor-core" : "CUDA-core");
    report += line;
    A43G_CUDA_TRY(cudaStreamSynchronize(st));
    return true;
}

template bool autotune<float>(GreenPlan const &, DevicePlan &, cudaStream_t, std::string &);
template bool autotune<double>(GreenPlan const &, DevicePlan &, cudaStream_t, std::string &);

} // namespace a43g
