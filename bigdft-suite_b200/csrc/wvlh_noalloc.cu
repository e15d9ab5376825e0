// Local Hamiltonian of one orbital without any device allocation.
//
// Some callers cannot call cudaMalloc at all: code running under a memory
// manager that owns every device allocation (a host program whose allocator
// hands out one fixed pool and fails any allocation made around it), and
// library layers that must not grow the device footprint behind their host's
// back.  For them this file gives one entry
// point that runs the same fused kernels as wvlh_locham_batched, with every
// table and all of its scratch (the P, Q/Z1 and Z2 planes and the energy
// partials) carved out of a file-scope static device array of fixed size.
// The caller passes only its own inputs and outputs.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/wvlh.h"
#include "wvlh_common.cuh"
#include "wvlh_internal.h"

namespace wvlh {
template <class T, class TIO>
cudaError_t launch_locham(const Plan &p, const TIO *psi, const TIO *pot, TIO *hpsi, T *scratch, double *part_pot,
                          double *part_kin, double *ekin, double *epot, int accumulate, cudaStream_t st,
                          cudaEvent_t *ev);
void set_last_error(int code);
}  // namespace wvlh

using namespace wvlh;

// The static scratch: 64 MiB on every device the entry point is used on, held
// until the process exits.  Host code never dereferences this symbol: its
// address on the current device is obtained with cudaGetSymbolAddress.
constexpr size_t kNoAllocBytes = size_t(64) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void *g_scratch_addr[kMaxDevices] = {nullptr};

// decoded segment {i0, i2, len, jj0} from 1-based keys (un-compress.f90:896-905)
__global__ void k_decode_segments(int n1, int n2, int nseg, const int32_t *__restrict__ keyg,
                                  const int32_t *__restrict__ keyv, int4 *__restrict__ seg)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nseg) return;
    const int j0 = keyg[2 * s], j1 = keyg[2 * s + 1];
    int ii = j0 - 1;
    const int i3 = ii / (n1 * n2);
    ii -= i3 * n1 * n2;
    const int i2 = ii / n1;
    seg[s] = make_int4(ii - i2 * n1, i2, j1 - j0 + 1, keyv[s] - 1);
}

// first segment of each coarse z-plane (keys are sorted by linear index)
__global__ void k_plane_ranges(int n12, int n3, int nseg, const int32_t *__restrict__ keyg, int *__restrict__ plane)
{
    const int i3 = blockIdx.x * blockDim.x + threadIdx.x;
    if (i3 > n3) return;
    int lo = 0, hi = nseg;  // first s with (keyg[2s]-1)/n12 >= i3
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if ((keyg[2 * mid] - 1) / n12 < i3) lo = mid + 1; else hi = mid;
    }
    plane[i3] = lo;
}

// work tables of one orbital: {0, G3} plane-kernel items, {0, n2} and {0, n2p}
// z-kernel tiles of the potential and kinetic chains
__global__ void k_work_lists(int G3, int n2, int n2p, int *pre13, int *pre2, int *pre2p)
{
    if (threadIdx.x == 0) {
        pre13[0] = 0;
        pre13[1] = G3;
        pre2[0] = 0;
        pre2[1] = n2;
        pre2p[0] = 0;
        pre2p[1] = n2p;
    }
}

inline size_t up256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace

extern "C" size_t wvlh_noalloc_capacity(void) { return kNoAllocBytes; }

extern "C" int wvlh_locham_noalloc(int precision, const int n[3], const int periodic[3], const double hgrid[3],
                                   int nseg_c, const int32_t *keyg_c, const int32_t *keyv_c, int nseg_f,
                                   const int32_t *keyg_f, const int32_t *keyv_f, const void *psi, const void *pot,
                                   void *hpsi, double *ekin, double *epot, void *stream)
{
    if ((precision != 32 && precision != 64) || !n || !periodic || !hgrid || !psi || !pot || !hpsi || !ekin ||
        !epot || nseg_c < 0 || nseg_f < 0 || (nseg_c && (!keyg_c || !keyv_c)) || (nseg_f && (!keyg_f || !keyv_f))) {
        set_last_error(WVLH_ERR_ARG);
        return WVLH_ERR_ARG;
    }
    int N[3], per[3];
    for (int k = 0; k < 3; ++k) {
        N[k] = n[k];
        per[k] = periodic[k] ? 1 : 0;
        if (N[k] < 1 || N[k] > 1024 || (per[k] && N[k] < 8)) {
            set_last_error(WVLH_ERR_ARG);
            return WVLH_ERR_ARG;
        }
    }
    // host-side validation of the keys (the same check as every other entry point)
    long long nvc = 0, nvf = 0;
    int rc = check_keys(N, nseg_c, keyg_c, keyv_c, &nvc);
    if (!rc) rc = check_keys(N, nseg_f, keyg_f, keyv_f, &nvf);
    if (rc) {
        set_last_error(rc);
        return rc;
    }
    const int G[3] = {2 * N[0], 2 * N[1], 2 * N[2]};
    int F[3], I[3];
    for (int k = 0; k < 3; ++k) {
        F[k] = fine_len(N[k], per[k]);
        I[k] = isf_len(N[k], per[k]);
    }
    const size_t es = precision == 32 ? 4 : 8;
    const int ntx0 = (I[0] + TX_ - 1) / TX_, nty0 = (I[1] + TY_ - 1) / TY_;
    const int ntx1 = (F[0] + TX_ - 1) / TX_, nty1 = (F[1] + TY_ - 1) / TY_;
    const int stride = (ntx0 * nty0 > ntx1 * nty1 + G[2]) ? ntx0 * nty0 : ntx1 * nty1 + G[2];
    const long long sP = (long long)G[2] * F[1] * F[0], sQ = (long long)G[2] * I[1] * I[0];
    // layout of the static array
    size_t off = 0;
    const size_t o_lr = off; off = up256(off + sizeof(LrDev));
    const size_t o_orb = off; off = up256(off + sizeof(OrbDev));
    const size_t o_kc = off; off = up256(off + 8 * (size_t)nseg_c + 4 * (size_t)nseg_c);
    const size_t o_kf = off; off = up256(off + 8 * (size_t)nseg_f + 4 * (size_t)nseg_f);
    const size_t o_sc = off; off = up256(off + 16 * (size_t)nseg_c);
    const size_t o_sf = off; off = up256(off + 16 * (size_t)nseg_f);
    const size_t o_pc = off; off = up256(off + 4 * (size_t)(N[2] + 1));
    const size_t o_pf = off; off = up256(off + 4 * (size_t)(N[2] + 1));
    const size_t o_w13 = off; off = up256(off + 2 * sizeof(int));
    const size_t o_w2 = off; off = up256(off + 2 * sizeof(int));
    const size_t o_w2p = off; off = up256(off + 2 * sizeof(int));
    const size_t o_pp = off; off = up256(off + 8 * (size_t)stride);
    const size_t o_pk = off; off = up256(off + 8 * (size_t)stride);
    const size_t o_scr = off; off = up256(off + es * (size_t)(2 * sP + sQ));
    if (off > kNoAllocBytes) {
        set_last_error(WVLH_ERR_TOO_LARGE);
        return WVLH_ERR_TOO_LARGE;
    }
    // plane buffers as the fused kernels lay them out (coarse_width, vec_pitch)
    const int W1 = coarse_width(N[0]), W2 = coarse_width(N[1]);
    const size_t width = (size_t)(W1 > F[0] ? (W1 > I[0] ? W1 : I[0]) : (F[0] > I[0] ? F[0] : I[0]));
    const size_t pitch = (size_t)vec_pitch((int)width);
    const size_t rows = (size_t)(W2 > F[1] ? (W2 > I[1] ? W2 : I[1]) : (F[1] > I[1] ? F[1] : I[1]));
    const size_t zl = (size_t)(G[2] > F[2] ? (G[2] > I[2] ? G[2] : I[2]) : (F[2] > I[2] ? F[2] : I[2]));
    // second plane buffer: P (F2 rows x pitch) or a transposed plane, each
    // pass's lines along x at the vec_pitch of its y length
    size_t planeB = (size_t)F[1] * pitch;
    const size_t uses[4] = {(size_t)F[0] * vec_pitch(W2), (size_t)I[0] * vec_pitch(F[1]),
                            (size_t)F[0] * vec_pitch(I[1]), (size_t)W1 * vec_pitch(F[1])};
    for (size_t u : uses) planeB = u > planeB ? u : planeB;
    int dev = 0, smax = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        set_last_error(WVLH_ERR_CUDA);
        return WVLH_ERR_CUDA;
    }
    if (cudaDeviceGetAttribute(&smax, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess || smax <= 1024) {
        set_last_error(WVLH_ERR_CUDA);
        return WVLH_ERR_CUDA;
    }
    if ((rows * pitch + planeB) * es > (size_t)smax - 1024 || 2 * zl * TX_ * TY_ * es > (size_t)smax - 1024) {
        set_last_error(WVLH_ERR_TOO_LARGE);
        return WVLH_ERR_TOO_LARGE;
    }
    // one-time set-up on this device: the device address of the static array,
    // kept for the life of the process (the library does not support a reset
    // of the device, which would reload its module, while it is loaded)
    unsigned char *base;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_addr[dev]) {
            void *a = nullptr;
            if (cudaGetSymbolAddress(&a, g_noalloc_scratch) != cudaSuccess || !a) {
                set_last_error(WVLH_ERR_CUDA);
                return WVLH_ERR_CUDA;
            }
            g_scratch_addr[dev] = a;
        }
        base = (unsigned char *)g_scratch_addr[dev];
    }
    cudaStream_t st = (cudaStream_t)stream;
    LrDev L;
    for (int k = 0; k < 3; ++k) {
        L.N[k] = N[k];
        L.per[k] = per[k];
        L.hgrid[k] = hgrid[k];
    }
    L.nseg_c = nseg_c;
    L.nseg_f = nseg_f;
    L.nvctr_c = (int)nvc;
    L.nvctr_f = (int)nvf;
    L.seg_c = (const int4 *)(base + o_sc);
    L.seg_f = (const int4 *)(base + o_sf);
    L.plane_c = (const int *)(base + o_pc);
    L.plane_f = (const int *)(base + o_pf);
    OrbDev O;
    O.lr = 0;
    O.pad = 0;
    O.psi = 0;
    O.pot = 0;
    O.sP = 0;
    O.sQ = sP;
    O.sZ = sP + sQ;
    O.c = 0.0;
    O.in_ptr = nullptr;
    O.out_ptr = nullptr;
    O.pot_ptr = nullptr;
    cudaError_t e = cudaSuccess;
#define NA_CK(x)                                  \
    do {                                          \
        if ((e = (x)) != cudaSuccess) {           \
            set_last_error(WVLH_ERR_CUDA);        \
            return WVLH_ERR_CUDA;                 \
        }                                         \
    } while (0)
    NA_CK(cudaMemcpyAsync(base + o_lr, &L, sizeof(L), cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(base + o_orb, &O, sizeof(O), cudaMemcpyHostToDevice, st));
    int32_t *dkc = (int32_t *)(base + o_kc), *dkf = (int32_t *)(base + o_kf);
    if (nseg_c) {
        NA_CK(cudaMemcpyAsync(dkc, keyg_c, 8 * (size_t)nseg_c, cudaMemcpyHostToDevice, st));
        NA_CK(cudaMemcpyAsync(dkc + 2 * nseg_c, keyv_c, 4 * (size_t)nseg_c, cudaMemcpyHostToDevice, st));
        k_decode_segments<<<(nseg_c + 255) / 256, 256, 0, st>>>(N[0], N[1], nseg_c, dkc, dkc + 2 * nseg_c,
                                                                (int4 *)(base + o_sc));
    }
    if (nseg_f) {
        NA_CK(cudaMemcpyAsync(dkf, keyg_f, 8 * (size_t)nseg_f, cudaMemcpyHostToDevice, st));
        NA_CK(cudaMemcpyAsync(dkf + 2 * nseg_f, keyv_f, 4 * (size_t)nseg_f, cudaMemcpyHostToDevice, st));
        k_decode_segments<<<(nseg_f + 255) / 256, 256, 0, st>>>(N[0], N[1], nseg_f, dkf, dkf + 2 * nseg_f,
                                                                (int4 *)(base + o_sf));
    }
    k_plane_ranges<<<(N[2] + 256) / 256, 256, 0, st>>>(N[0] * N[1], N[2], nseg_c, dkc, (int *)(base + o_pc));
    k_plane_ranges<<<(N[2] + 256) / 256, 256, 0, st>>>(N[0] * N[1], N[2], nseg_f, dkf, (int *)(base + o_pf));
    k_work_lists<<<1, 32, 0, st>>>(G[2], ntx0 * nty0, ntx1 * nty1, (int *)(base + o_w13), (int *)(base + o_w2),
                                   (int *)(base + o_w2p));
    NA_CK(cudaGetLastError());
    // the launch plan lives on the host stack; its device tables point into the static array
    Plan p;
    p.nlr = 1;
    p.norb = 1;
    p.all_periodic = per[0] && per[1] && per[2];
    p.d_lr = (LrDev *)(base + o_lr);
    p.d_orb = (OrbDev *)(base + o_orb);
    p.d_pre13 = (int *)(base + o_w13);
    p.d_pre2 = (int *)(base + o_w2);
    p.d_pre2p = (int *)(base + o_w2p);
    p.n_work13 = G[2];
    p.n_work2 = ntx0 * nty0;
    p.n_work2p = ntx1 * nty1;
    p.part_stride = stride;
    p.plane_elems = (long long)(rows * pitch);
    {
        const long long len = (long long)width, ab = (long long)(rows * pitch + planeB);
        p.plane_threads[0] = choose_plane_threads({PlaneShape{(long long)rows, len, ab * 4, 1}}, true);
        p.plane_threads[1] = choose_plane_threads({PlaneShape{(long long)rows, len, ab * 8, 1}}, false);
    }
    p.planeB_elems = (long long)planeB;
    p.scratch_elems = 2 * sP + sQ;
    p.smem13[0] = (rows * pitch + planeB) * 4;
    p.smem13[1] = (rows * pitch + planeB) * 8;
    p.smem2[0] = 2 * zl * TX_ * TY_ * 4;
    p.smem2[1] = 2 * zl * TX_ * TY_ * 8;
    // the energy partials are cleared by the launcher; P, Q/Z1, Z2 are fully
    // overwritten before they are read, so stale contents of an earlier call
    // never leak into this one
    if (precision == 64)
        e = launch_locham<double, double>(p, (const double *)psi, (const double *)pot, (double *)hpsi,
                                          (double *)(base + o_scr), (double *)(base + o_pp), (double *)(base + o_pk),
                                          ekin, epot, 0, st, nullptr);
    else
        e = launch_locham<float, float>(p, (const float *)psi, (const float *)pot, (float *)hpsi,
                                        (float *)(base + o_scr), (double *)(base + o_pp), (double *)(base + o_pk),
                                        ekin, epot, 0, st, nullptr);
    NA_CK(e);
#undef NA_CK
    return WVLH_OK;
}
