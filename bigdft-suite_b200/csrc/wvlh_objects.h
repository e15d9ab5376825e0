// Objects shared by the host-side translation units of the library: the
// grow-only device buffer, the context and the resident region.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../../include/wvlh.h"
#include "wvlh_internal.h"

namespace wvlh {

// grow-only device buffer
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    int ensure(size_t b)
    {
        if (b <= bytes) return WVLH_OK;
        if (p) {
            // kernels queued earlier may still read the old buffer
            cudaDeviceSynchronize();
            cudaFree(p);
        }
        p = nullptr;
        bytes = 0;
        if (cudaMalloc(&p, b) != cudaSuccess) return WVLH_ERR_NOMEM;
        bytes = b;
        return WVLH_OK;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
};

}  // namespace wvlh

struct wvlh_ctx;
namespace wvlh {
// frees the Poisson solver's plans and buffers of a context (wvlh_psolver.cu)
void psolver_release(const wvlh_ctx *ctx);
}  // namespace wvlh

// the C ABI's opaque handles (global names, as include/wvlh.h declares them)
struct wvlh_ctx {
    int device = 0;
    cudaStream_t stream = 0;
    wvlh::DevBuf cg_r, cg_d, cg_ad, cg_scal, den_part, ov_work;
    // optional per-kernel timing of the fused locham (K1, K2, K3, reduction)
    int timing = 0;
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    double kernel_ms[4] = {0, 0, 0, 0};
    long long timed_calls = 0;
    wvlh::DevBuf scratch, part_pot, part_kin, io_psi, io_pot, io_hpsi, io_e, plain[4], dotpart;
    // tables of the orbital batches (wvlh_batch_create_orbitals): rewritten in
    // stream order by each new batch, whose generation number it records
    wvlh::DevBuf arena;
    unsigned long long arena_gen = 0;
    wvlh::DevBuf wp_runs;  // compressed scalar products: one run per b segment
    // host-buffer path: an upload stream and a download stream around the
    // context's stream, with per-chunk events (uploaded, computed)
    cudaStream_t aux = nullptr, aux2 = nullptr;
    cudaEvent_t ev_a = nullptr;
    std::vector<cudaEvent_t> ev_in, ev_cmp;
};

// One localisation region: its box and its keys, validated once and kept on
// the device in two forms: decoded {i0, i2, len, jj0} segments with per-plane
// ranges (fused kernels) and the raw 1-based keys (one-pass-per-kernel path).
struct wvlh_region {
    int device = 0;
    wvlh::LrDev lr{};
    const uint32_t *keyg_c = nullptr, *keyv_c = nullptr, *keyg_f = nullptr, *keyv_f = nullptr;
    double hgrid[3] = {0, 0, 0};
    void *mem = nullptr;  // one device block holding all of the above
};

