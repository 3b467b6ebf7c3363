// Upload of a host plan to the device and the derived neighbour table.
#include "device.cuh"

#include <algorithm>
#include <cstdlib>
#include <cstring>

namespace a43g {

bool DeviceBuffer::alloc(size_t n) {
    if (n <= bytes && ptr) return true;
    release();
    if (0 == n) return true;
    cudaError_t const e = cudaMalloc(&ptr, n);
    if (cudaSuccess != e) {
        ptr = nullptr; bytes = 0;
        set_error(std::string("cudaMalloc of ") + std::to_string(n) + " bytes: " + cudaGetErrorString(e));
        return false;
    }
    bytes = n;
    return true;
}

void DeviceBuffer::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr; bytes = 0;
}

namespace {

template <typename T>
bool put(DeviceBuffer &b, std::vector<T> const &v) {
    size_t const n = v.size()*sizeof(T);
    if (!b.alloc(std::max<size_t>(n, 16))) return false;
    if (n) A43G_CUDA_TRY(cudaMemcpy(b.ptr, v.data(), n, cudaMemcpyHostToDevice));
    return true;
}

// Neighbour of every block along each direction, read off the finite-difference lists:
// consecutive list entries are neighbours; the entries before the first and after the last
// cube are the halo (0: zero cube, negative: periodic image, src/kinetic_plan.cxx:153-179).
std::vector<int32_t> neighbour_table(GreenPlan const &hp) {
    size_t const nnzb = hp.nnzb();
    std::vector<int32_t> nbr(6*nnzb, -1);
    for (int dd = 0; dd < 3; ++dd) {
        auto const &K = hp.kinetic[dd];
        for (uint32_t il = 0; il < K.nlists(); ++il) {
            int32_t const *L = &K.entry[K.start[il]];
            int const len = int(K.start[il + 1] - K.start[il]);
            int n = 0;
            while (kNhalo + n < len && L[kNhalo + n] > 0) ++n;
            for (int i = 0; i < n; ++i) {
                int32_t const b = L[kNhalo + i] - 1;
                auto code = [](int32_t entry) -> int32_t {
                    if (entry > 0) return entry - 1;          // plain neighbour
                    if (entry < 0) return -(-entry - 1) - 2;  // periodic image
                    return -1;                                 // zero cube
                };
                nbr[6*size_t(b) + 2*dd + 0] = code(L[kNhalo + i - 1]);
                nbr[6*size_t(b) + 2*dd + 1] = code(L[kNhalo + i + 1]);
            }
        }
    }
    return nbr;
}

} // namespace

bool upload_plan(GreenPlan const &hp, DevicePlan &dp) {
    if (!prepare_simt_kernels() || !prepare_tc_kernels() || !prepare_local_kernels()) return false;
    dp.nnzb = uint32_t(hp.nnzb()); dp.nRows = hp.nRows; dp.nCols = hp.nCols;
    dp.nAtoms = hp.nAtoms; dp.nAI = hp.nAtomImages;
    dp.ncoeffI = uint32_t(hp.ncoeff_images()); dp.ncoeffA = uint32_t(hp.ncoeff_atoms());
    dp.lmax_max = -1;
    for (auto l : hp.AtomImageLmax) dp.lmax_max = std::max(dp.lmax_max, int(l));
    bool all4 = true;
    for (int d = 0; d < 3; ++d) {
        dp.FD_range[d] = hp.kinetic[d].FD_range;
        dp.prefactor[d] = hp.kinetic[d].prefactor;
        dp.nlists[d] = hp.kinetic[d].nlists();
        all4 = all4 && (dp.FD_range[d] >= 1 && dp.FD_range[d] != 8);
        dp.grid[d] = hp.grid_spacing_dyadic[d];
    }
    dp.grid[3] = hp.grid_spacing_dyadic[3];
    dp.fused_local = all4;
    dp.max_zline = 0;
    {
        auto const &K = hp.kinetic[2];
        for (uint32_t il = 0; il < K.nlists(); ++il) {
            uint32_t const len = K.start[il + 1] - K.start[il];
            dp.max_zline = std::max(dp.max_zline, len > 2*kNhalo ? len - 2*kNhalo : 0u);
        }
    }

    if (!put(dp.veff_index, hp.veff_index)) return false;
    if (!put(dp.nbr, neighbour_table(hp))) return false;
    for (int d = 0; d < 3; ++d) {
        if (!put(dp.lists_start[d], hp.kinetic[d].start)) return false;
        if (!put(dp.lists[d], hp.kinetic[d].entry)) return false;
    }
    if (!put(dp.colindx, hp.colindx)) return false;
    if (!put(dp.rowindx, hp.rowindx)) return false;
    if (!put(dp.rowCubePos, hp.rowCubePos)) return false;
    // dyadic sparsity
    std::vector<uint32_t> ps, pc; std::vector<uint64_t> po;
    for (uint32_t s = 0; s < hp.nCols; ++s) {
        po.push_back(pc.size());
        auto const &c = hp.SHOprj[s];
        if (c.start.empty()) ps.insert(ps.end(), hp.nAtomImages + 1, 0u);
        else ps.insert(ps.end(), c.start.begin(), c.start.end());
        pc.insert(pc.end(), c.col.begin(), c.col.end());
    }
    if (!put(dp.prj_start, ps) || !put(dp.prj_col, pc) || !put(dp.prj_coloff, po)) return false;
    if (!put(dp.add_start, hp.SHOadd.start) || !put(dp.add_col, hp.SHOadd.col)) return false;
    if (!put(dp.sum_start, hp.SHOsum.start) || !put(dp.sum_col, hp.SHOsum.col)) return false;
    if (!put(dp.img_pos, hp.AtomImagePos) || !put(dp.img_lmax, hp.AtomImageLmax)) return false;
    if (!put(dp.img_starts, hp.AtomImageStarts)) return false;
    if (!put(dp.atom_starts, hp.AtomStarts) || !put(dp.atom_lmax, hp.AtomLmax)) return false;
    if (!put(dp.atom_mat_off, hp.AtomMatOffset)) return false;
    if (!put(dp.grid_dev, std::vector<double>(dp.grid, dp.grid + 4))) return false;
    for (int L = 0; L < 8; ++L) {
        std::vector<uint32_t> imgs;
        for (uint32_t a = 0; a < hp.nAtomImages; ++a) if (hp.AtomImageLmax[a] == L) imgs.push_back(a);
        dp.img_group[L].count = uint32_t(imgs.size());
        if (!put(dp.img_group[L].images, imgs)) return false;
    }
    if (dp.lmax_max > 7) { set_error("projector basis sizes above numax 7 are not supported"); return false; }
    if (!build_prj_items(hp, dp)) return false;
    dp.table_stride = (hp.table_lmax + 1)*12;
    if (!put(dp.slot_H, hp.slot_H) || !put(dp.slot_mask, hp.slot_mask)) return false;
    if (!put(dp.slot_H32, std::vector<float>(hp.slot_H.begin(), hp.slot_H.end()))) return false;
    if (!put(dp.prj_slot, hp.prj_slot) || !put(dp.add_slot, hp.add_slot)) return false;
    {   // one 16-byte record per addition pair, so the kernel needs no dependent index loads
        std::vector<uint32_t> info(4*size_t(hp.SHOadd.nnz()), 0u);
        for (size_t k = 0; k < hp.SHOadd.nnz(); ++k) {
            uint32_t const a = hp.SHOadd.col[k];
            info[4*k + 0] = hp.add_slot[k];
            info[4*k + 1] = hp.AtomImageStarts[a];
            info[4*k + 2] = uint32_t(hp.AtomImageLmax[a]);
        }
        if (!put(dp.add_info, info)) return false;
    }
    if (!put(dp.subset_dev, hp.subset)) return false;
    {   // blocks of every source, in block order
        std::vector<uint32_t> start(hp.nCols + 1, 0), blocks(hp.nnzb());
        for (size_t b = 0; b < hp.nnzb(); ++b) ++start[hp.colindx[b] + 1];
        for (uint32_t c = 0; c < hp.nCols; ++c) start[c + 1] += start[c];
        std::vector<uint32_t> fill(start.begin(), start.end() - 1);
        for (size_t b = 0; b < hp.nnzb(); ++b) blocks[fill[hp.colindx[b]]++] = uint32_t(b);
        dp.max_src_blocks = 0;
        for (uint32_t c = 0; c < hp.nCols; ++c) dp.max_src_blocks = std::max(dp.max_src_blocks, start[c + 1] - start[c]);
        if (!put(dp.src_start, start) || !put(dp.src_blocks, blocks)) return false;
        if (!put(dp.src_active, std::vector<uint8_t>(std::max<size_t>(hp.nCols, 1), uint8_t(1)))) return false;
        dp.retire = false;
    }
    dp.npairs = hp.npairs;
    dp.nsrc_pair = (hp.npairs > 1) ? hp.nsrc_pair : hp.nCols;
    dp.mat_stride = hp.AtomMatrices.size();
    if (!put(dp.dev_error, std::vector<int32_t>(4, 0))) return false;
    {
        // FP32 projector: SIMT (default) or the tensor cores ("tc"); the FP64 path is always SIMT
        char const *e = std::getenv("A43G_PROJECTOR");
        dp.use_tc = (e && 0 == std::strcmp(e, "tc"));
        // FP32 local kernel: y-"pencils" (default), pencils with "staged" neighbour cubes, "rows"
        // with loads ahead or "plain" rows
        char const *l = std::getenv("A43G_LOCAL");
        dp.local_variant = (l && 0 == std::strcmp(l, "plain")) ? 1 : ((l && 0 == std::strcmp(l, "rows")) ? 0 :
                           ((l && 0 == std::strcmp(l, "staged")) ? 3 : 2));
        // FP64 local kernel: "pencils" (default) or "rows"
        char const *l64 = std::getenv("A43G_LOCAL64");
        dp.local64_pencils = !(l64 && 0 == std::strcmp(l64, "rows"));
        // FP64 addition: z-orders "unrolled" (default) or "rolled"
        char const *a64 = std::getenv("A43G_ADD64");
        dp.add64_unrolled = !(a64 && 0 == std::strcmp(a64, "rolled"));
        // atom-matrix chain: one kernel (default) or "three" (collect, multiply, broadcast)
        char const *ac = std::getenv("A43G_ATOM_CHAIN");
        dp.atom_chain3 = (ac && 0 == std::strcmp(ac, "three"));
    }
    if (!dp.aac.alloc(std::max<size_t>(16, size_t(dp.ncoeffA)*dp.nCols*128*sizeof(double)))) return false;
    if (!dp.cadd.alloc(std::max<size_t>(16, size_t(dp.ncoeffA)*dp.nCols*128*sizeof(double)))) return false;
    dp.uploaded = true;
    dp.values_dirty = true;
    return upload_values(hp, dp);
}

bool build_prj_items(GreenPlan const &hp, DevicePlan &dp) {
    uint32_t const chunk = std::max<uint32_t>(1, dp.prj_chunk);
    std::vector<uint32_t> items[8], items8[8];
    uint32_t groups[8] = {0}, parts[8] = {0};
    for (uint32_t s = 0; s < hp.nCols; ++s) {
        auto const &c = hp.SHOprj[s];
        if (c.start.empty()) continue;
        for (uint32_t a = 0; a < hp.nAtomImages; ++a) {
            int const L = hp.AtomImageLmax[a];
            uint32_t const k0 = c.start[a], k1 = c.start[a + 1];
            if (k0 >= k1) continue;
            uint32_t const n = (k1 - k0 + chunk - 1)/chunk, first = uint32_t(items[L].size()/4);
            uint32_t const part = (n > 1) ? parts[L] : 0u;
            for (uint32_t k = k0; k < k1; k += chunk) {
                uint32_t const it[4] = {a, s, k, std::min(k + chunk, k1)};
                items[L].insert(items[L].end(), it, it + 4);
                uint32_t const it8[8] = {a, s, k, std::min(k + chunk, k1), first, n, groups[L], part};
                items8[L].insert(items8[L].end(), it8, it8 + 8);
            }
            ++groups[L];
            if (n > 1) parts[L] += n;
        }
    }
    for (int L = 0; L < 8; ++L) {
        auto &g = dp.prj_items[L];
        g.count = uint32_t(items[L].size()/4);
        g.part_items = parts[L];
        if (!put(g.items, items[L]) || !put(g.items8, items8[L])) return false;
        if (!put(g.tickets, std::vector<uint32_t>(std::max<uint32_t>(groups[L], 1), 0u))) return false;
    }
    return true;
}

bool ensure_prj_part(DevicePlan &dp, size_t elem_bytes) {
    size_t n = 16;
    for (int L = 0; L < 8; ++L)
        n = std::max(n, size_t(dp.prj_items[L].part_items)*size_t(((L + 1)*(L + 2)*(L + 3))/6)*128*elem_bytes);
    return dp.prj_part.alloc(n);
}

bool upload_values(GreenPlan const &hp, DevicePlan &dp) {
    if (!put(dp.Vcell64, hp.Vcell)) return false;
    std::vector<float> v32(hp.Vcell.begin(), hp.Vcell.end());
    if (!put(dp.Vcell32, v32)) return false;
    if (hp.npairs > 1) {
        // batch plan: image phases and atom matrices [pair][...], energies and phases per pair
        if (!put(dp.atom_mat, hp.pair_mats)) return false;
        if (!put(dp.img_phase, hp.pair_img_phase)) return false;
        std::vector<double> a64(14*size_t(hp.npairs));
        std::vector<float> a32(14*size_t(hp.npairs));
        for (uint32_t p = 0; p < hp.npairs; ++p) {
            a64[14*p] = hp.pair_E[2*p]; a64[14*p + 1] = hp.pair_E[2*p + 1];
            for (int k = 0; k < 12; ++k) a64[14*p + 2 + k] = hp.pair_phase[12*size_t(p) + k];
        }
        for (size_t k = 0; k < a64.size(); ++k) a32[k] = float(a64[k]);
        if (!put(dp.pair_args64, a64) || !put(dp.pair_args32, a32)) return false;
    } else {
        if (!put(dp.atom_mat, hp.AtomMatrices)) return false;
        if (!put(dp.img_phase, hp.AtomImagePhase)) return false;
    }
    std::memcpy(dp.phase, hp.phase, sizeof(dp.phase));
    dp.E_re = hp.E_re; dp.E_im = hp.E_im;
    dp.values_dirty = false;
    return true;
}

bool ensure_dyadic_scratch(DevicePlan &dp, size_t elem_bytes) {
    size_t const n = std::max<size_t>(16, size_t(dp.ncoeffI)*dp.nCols*128*elem_bytes);
    if (dp.apc.bytes >= n && dp.cad.bytes >= n) return true;
    return dp.apc.alloc(n) && dp.cad.alloc(n);
}

// flop count of one application as the reference counts it (include/green_potential.hxx:171-177,
// include/green_kinetic.hxx:381, include/dyadic_plan.hxx:93-103), R1C2 = 2, Noco = 1
double action_flops(GreenPlan const &hp, int /*real_bytes*/) {
    double const nnzb = double(hp.nnzb());
    double f = (1 + 2*(0 != hp.E_im))*nnzb*4096*2;
    for (int d = 0; d < 3; ++d) {
        int const nFD = (hp.kinetic[d].FD_range >= 1 && hp.kinetic[d].nlists() > 0) ? hp.kinetic[d].FD_range : 0;
        f += nnzb*(2*nFD + 1)*2*4096*2;
    }
    if (hp.nAtomImages > 0 && hp.nCols > 0) {
        auto flop_prj_add = [](int L) {
            return 2*(64*(L + 1) + 16*(((L + 1)*(L + 2))/2) + 4*(((L + 1)*(L + 2)*(L + 3))/6));
        };
        double gen = 0, addc = 0, mul = 0, sum = 0;
        for (uint32_t k = 0; k < hp.SHOadd.nnz(); ++k) {
            int const L = hp.AtomImageLmax[hp.SHOadd.col[k]];
            addc += 64.0*flop_prj_add(L);
            gen += 12.0*(7 + 4*L);
        }
        for (uint32_t ia = 0; ia < hp.nAtoms; ++ia) { double const n = nsho(hp.AtomImageLmax[ia]); mul += n*n; }
        mul *= 2.0*hp.nCols*64;
        if (hp.nAtomImages > hp.nAtoms) {
            for (uint32_t a = 0; a < hp.nAtomImages; ++a) sum += nsho(hp.AtomImageLmax[a]);
            sum *= 2.0*hp.nCols*64;
        }
        f += mul*4 + 2*sum*4 + 2*gen + 2*addc*2;
    }
    return f;
}

} // namespace a43g
