// validate.cu -- consistency checks of the device state on the host (the race detector of a
// Gauss-Seidel on a colouring: no body may appear twice in one colour) and a self-test of the
// bounded device waits.
//
// pe has no counterpart beyond its debug assertions (pe_INTERNAL_ASSERT, compiled out under
// NDEBUG); these checks run only when called.
#include <algorithm>
#include <vector>

#include "internal.cuh"
#include "validate_host.h"

namespace peb {

namespace {

// Waits for a flag nothing sets, with the bounded poll of the grid barriers: after `polls`
// polls it records DERR_TIMEOUT and returns, leaving the context usable.
__global__ void k_wait_never(const unsigned int *flag, unsigned long long polls, int32_t *err) {
    if (threadIdx.x != 0) return;
    unsigned long long spins = 0;
    for (;;) {
        unsigned int v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(flag) : "memory");
        if (v != 0u) return;
        if (++spins > 64) __nanosleep(64);
        if (spins > polls) {
            atomicOr(err, DERR_TIMEOUT);
            return;
        }
    }
}

}  // namespace

// HCSITS: every colour of the last step's contact order holds each body at most once.
int validate_coloring(Ctx *c, int64_t *bad) {
    const NbgsBuf &nb = c->nb;
    const int64_t nc = c->last_ncontacts;
    const int ncol = c->last_ncolors;
    if (nc <= 0 || ncol <= 0 || !nb.cache || !nb.color_start) return PE_B200_OK;
    std::vector<int32_t> ids(2 * nc);
    PEB_CUDA(c, cudaStreamSynchronize(c->stream));
    // a queued step left its colour offsets on the device only
    if (nb.on_device && nb.cstart_dev) {
        PEB_CUDA(c, cudaMemcpyAsync(nb.color_start, nb.cstart_dev, (ncol + 1) * sizeof(int32_t),
                                    cudaMemcpyDeviceToHost, c->stream));
        PEB_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    PEB_CUDA(c, cudaMemcpyAsync(ids.data(), nbgs_ids_ptr(c), nc * sizeof(int2), cudaMemcpyDeviceToHost, c->stream));
    PEB_CUDA(c, cudaStreamSynchronize(c->stream));
    *bad += coloring_problems(c->n + c->mb.m, nc, ids.data(), ncol, nb.color_start);
    return PE_B200_OK;
}

// DEM lists: the CSR lists of the last rebuild (skipped when it overflowed: lists incomplete)
int validate_lists(Ctx *c, int64_t *bad) {
    const ListBuf &L = c->nl;
    const int64_t n = c->n;
    // lists exist once a list step has run (scenes with moving boxes use the cell grid)
    if (!L.enabled || !L.warm || c->mb.m > 0 || n == 0 || !L.start || !L.flags) return PE_B200_OK;
    PEB_CUDA(c, cudaStreamSynchronize(c->stream));
    int32_t flags[4];
    PEB_CUDA(c, cudaMemcpyAsync(flags, L.flags, sizeof flags, cudaMemcpyDeviceToHost, c->stream));
    PEB_CUDA(c, cudaStreamSynchronize(c->stream));
    if (flags[1] != 0) return PE_B200_OK;
    std::vector<int32_t> start(n + 1), uid(n);
    PEB_CUDA(c, cudaMemcpyAsync(start.data(), L.start, (n + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    PEB_CUDA(c, cudaMemcpyAsync(uid.data(), c->cur.uid, n * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    PEB_CUDA(c, cudaStreamSynchronize(c->stream));
    const int64_t m = std::min<int64_t>(std::max<int64_t>(start[n], 0), L.cap);
    std::vector<int32_t> idx(std::max<int64_t>(m, 1));
    if (m) PEB_CUDA(c, cudaMemcpyAsync(idx.data(), L.idx, m * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    PEB_CUDA(c, cudaStreamSynchronize(c->stream));
    *bad += list_problems(n, L.cap, start.data(), idx.data(), uid.data());
    return PE_B200_OK;
}

int selftest_timeout(Ctx *c, int64_t polls) {
    unsigned int *flag = nullptr;
    PEB_CUDA(c, dmalloc(c, &flag, sizeof(unsigned int)));
    cudaError_t e = cudaMemsetAsync(flag, 0, sizeof(unsigned int), c->stream);
    if (e == cudaSuccess) {
        k_wait_never<<<1, 32, 0, c->stream>>>(flag, (unsigned long long)polls, c->d_err);
        e = cudaGetLastError();
        c->launches++;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    dfree(c, flag);
    if (e != cudaSuccess) return cuda_err(c, e, "timeout self-test");
    return PE_B200_OK;
}

}  // namespace peb
