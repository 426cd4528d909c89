// rebuild.cu -- the neighbour-list rebuild of the DEM step as one persistent kernel.
//
// One cooperative launch per step.  Unless the previous force kernel requested a rebuild (a
// sphere has moved skin/2 since the last one) every block returns after reading one flag, so a
// step without a rebuild pays a single short launch; the kernel is launched to be scheduled
// while the one before it finishes (programmatic dependent launch).  The stages are in
// rebuild.cuh.  The list step of a single-stream context runs the rebuild and the contact
// forces in one kernel instead (dem.cu k_rebuild_contacts); this kernel serves the others.
#include <algorithm>

#include "rebuild.cuh"

namespace peb {

namespace {

template <typename VT>
__global__ void __launch_bounds__(kRbBlock) k_rebuild(RebuildArgs<VT> a) {
    // scheduled while the previous force kernel finishes; its flag is read after it has
    pdl_wait();
    if (!a.flags[0]) {  // uniform: no rebuild requested; the force kernel may start
        // the force kernels read the current state (flags[4]: the step rebuilt, read the copy)
        if (blockIdx.x == 0 && threadIdx.x == 0) a.flags[4] = 0;
        pdl_trigger();
        return;
    }
    rebuild_stages(a);
}

template <typename VT>
int launch_rebuild(Ctx *c) {
    ListBuf &L = c->nl;
    static thread_local int occ_cache[2] = {0, 0};
    int &occ = occ_cache[sizeof(VT) == 8 ? 1 : 0];
    if (occ == 0) {
        PEB_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_rebuild<VT>, kRbBlock, 0));
        if (occ < 1) return set_err(c, PE_B200_ERR_CUDA, "rebuild kernel cannot be resident");
    }
    RebuildArgs<VT> a;
    unsigned grid = 0;
    int rc = rebuild_setup<VT>(c, occ, a, &grid);
    if (rc) return rc;
    // cooperative, and scheduled while the force kernel before it finishes; without the early
    // start if the driver refuses the pair of attributes
    if (!L.rebuild_pdl_off) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(grid);
        cfg.blockDim = dim3(kRbBlock);
        cfg.stream = c->stream;
        cudaLaunchAttribute at[2];
        at[0].id = cudaLaunchAttributeCooperative;
        at[0].val.cooperative = 1;
        at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[1].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = at;
        cfg.numAttrs = 2;
        if (cudaLaunchKernelEx(&cfg, k_rebuild<VT>, a) == cudaSuccess) {
            c->launches++;
            return PE_B200_OK;
        }
        cudaGetLastError();
        L.rebuild_pdl_off = true;
    }
    void *args[] = {&a};
    PEB_CUDA(c, cudaLaunchCooperativeKernel((const void *)k_rebuild<VT>, dim3(grid),
                                            dim3(kRbBlock), args, 0, c->stream));
    c->launches++;
    return PE_B200_OK;
}

}  // namespace

int dem_list_rebuild_persistent(Ctx *c) {
    return (c->p.precision == PE_B200_FP64) ? launch_rebuild<double>(c) : launch_rebuild<float>(c);
}

}  // namespace peb
