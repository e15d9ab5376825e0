// Batched ABI: contexts, regions (validated and decoded keys of one
// localisation region, resident on the device), batch plans (work tables) and
// the batched local-Hamiltonian, density, preconditioner and overlap entry
// points.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "../../include/wvlh.h"
#include "wvlh_common.cuh"
#include "wvlh_internal.h"
#include "wvlh_objects.h"
#include "wvlh_plain.h"
#include "wvlh_tma.cuh"

#include <cudaTypedefs.h>

namespace wvlh {
template <class T, class TIO>
cudaError_t launch_locham(const Plan &p, const TIO *psi, const TIO *pot, TIO *hpsi, T *scratch, double *part_pot,
                          double *part_kin, double *ekin, double *epot, int accumulate, cudaStream_t st,
                          cudaEvent_t *ev);
cudaError_t fma_probe(int precision, int iters, float *ms, double *flops, cudaStream_t st);
long long plane_tmp_elems(const Plan &p, int fp);
void set_last_error(int code);
}  // namespace wvlh

using namespace wvlh;

struct wvlh_batch {
    wvlh_ctx *ctx = nullptr;
    Plan plan;
    std::vector<int64_t> pot_off;
    bool density_ok = true;                  // orbitals sharing a density grid share its region
    std::vector<const wvlh_region *> lr;     // region of each plan region index
    std::vector<wvlh_region *> own_regions;  // regions made by wvlh_batch_create
    // orbital batches: per-orbital device buffers, tables in the context arena
    bool orbital_mode = false;
    bool can_locham = true, can_locden = true;
    unsigned long long arena_gen = 0;
    void *mem = nullptr;  // owned table block (wvlh_batch_create)
    // host-buffer path: sub-batches over consecutive orbital ranges (made on first use)
    std::vector<wvlh_batch *> chunks;
    std::vector<int> chunk_o0;
};

static void apply_tuned(Plan &p);

static int fail(int code)
{
    set_last_error(code);
    return code;
}

#define CK(x)                                                      \
    do {                                                           \
        cudaError_t e_ = (x);                                      \
        if (e_ != cudaSuccess) {                                   \
            fprintf(stderr, "wvlh: %s\n", cudaGetErrorString(e_)); \
            return fail(WVLH_ERR_CUDA);                            \
        }                                                          \
    } while (0)

// Host image of a set of device tables at 256-byte aligned offsets of one
// device block; the pointers are set once the block's address is known.
struct Packer {
    std::vector<unsigned char> img;
    std::vector<std::pair<void **, size_t>> fix;
    template <class T, class P>
    void add(const std::vector<T> &v, P **dst)
    {
        static_assert(sizeof(T) == sizeof(P), "table element type");
        *dst = nullptr;
        if (v.empty()) return;
        const size_t off = (img.size() + 255) & ~size_t(255);
        img.resize(off + v.size() * sizeof(T));
        memcpy(img.data() + off, v.data(), v.size() * sizeof(T));
        fix.emplace_back(reinterpret_cast<void **>(const_cast<std::remove_const_t<P> **>(dst)), off);
    }
    void place(void *base)
    {
        for (auto &f : fix) *f.first = static_cast<unsigned char *>(base) + f.second;
    }
};

extern "C" int wvlh_ctx_create(int device, wvlh_ctx **ctx)
{
    if (!ctx) return fail(WVLH_ERR_ARG);
    CK(cudaSetDevice(device));
    wvlh_ctx *c = new wvlh_ctx();
    c->device = device;
    *ctx = c;
    return WVLH_OK;
}

extern "C" int wvlh_ctx_destroy(wvlh_ctx *ctx)
{
    if (!ctx) return WVLH_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (DevBuf *b : {&ctx->scratch, &ctx->part_pot, &ctx->part_kin, &ctx->io_psi, &ctx->io_pot, &ctx->io_hpsi,
                      &ctx->io_e, &ctx->dotpart, &ctx->cg_r, &ctx->cg_d, &ctx->cg_ad, &ctx->cg_scal, &ctx->den_part,
                      &ctx->ov_work, &ctx->arena, &ctx->wp_runs})
        b->release();
    for (auto &b : ctx->plain) b.release();
    for (auto &e : ctx->ev)
        if (e) cudaEventDestroy(e);
    if (ctx->ev_a) cudaEventDestroy(ctx->ev_a);
    for (cudaEvent_t e : ctx->ev_in) cudaEventDestroy(e);
    for (cudaEvent_t e : ctx->ev_cmp) cudaEventDestroy(e);
    for (cudaStream_t st : {ctx->aux, ctx->aux2})
        if (st) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
    psolver_release(ctx);
    delete ctx;
    return WVLH_OK;
}

extern "C" int wvlh_ctx_set_stream(wvlh_ctx *ctx, void *stream)
{
    if (!ctx) return fail(WVLH_ERR_ARG);
    ctx->stream = (cudaStream_t)stream;
    return WVLH_OK;
}

extern "C" int wvlh_ctx_synchronize(wvlh_ctx *ctx)
{
    if (!ctx) return fail(WVLH_ERR_ARG);
    CK(cudaStreamSynchronize(ctx->stream));
    return WVLH_OK;
}

namespace wvlh {
// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library)
bool encode_tile_map(CUtensorMap *map, const void *base, int elem_bytes, long long W, long long H, long long Z,
                     long long norb, long long orb_stride_elems)
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool looked = false;
    if (!looked) {
        looked = true;
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)f;
        cudaGetLastError();
    }
    if (!fn || Z > 256 || Z < 1 || W < 1 || H < 1 || norb < 1) return false;
    const long long rowb = W * elem_bytes, planeb = rowb * H, orbb = orb_stride_elems * elem_bytes;
    // strides and the base address must be multiples of 16 bytes
    if ((rowb % 16) || (planeb % 16) || (orbb % 16) || ((uintptr_t)base % 16)) return false;
    const cuuint64_t dim[4] = {(cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)Z, (cuuint64_t)norb};
    const cuuint64_t stride[3] = {(cuuint64_t)rowb, (cuuint64_t)planeb, (cuuint64_t)orbb};
    const cuuint32_t box[4] = {(cuuint32_t)TX_, (cuuint32_t)TY_, (cuuint32_t)Z, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = fn(map, elem_bytes == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4,
                          const_cast<void *>(base), dim, stride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}
}  // namespace wvlh

// Validate the reference's 1-based keys of one region and decode them into
// {i0, i2, len, jj0} plus per-plane segment ranges (wavelib/un-compress.f90:896-905).
static int decode_keys(const int *N, int nseg, const int32_t *keyg, const int32_t *keyv, std::vector<int4> &seg,
                       std::vector<int> &plane, int &nvctr)
{
    const long long n12 = (long long)N[0] * N[1];
    if (nseg > 0 && (!keyg || !keyv)) return WVLH_ERR_ARG;
    if (check_keys(N, nseg, keyg, keyv, nullptr)) return WVLH_ERR_KEYS;
    seg.resize(nseg);
    plane.assign(N[2] + 1, nseg);
    long long cum = 0;
    int cur_plane = 0;
    for (int s = 0; s < nseg; ++s) {
        const long long j0 = keyg[2 * s], j1 = keyg[2 * s + 1];
        long long ii = j0 - 1;
        const int i3 = (int)(ii / n12);
        ii -= (long long)i3 * n12;
        const int i2 = (int)(ii / N[0]);
        const int i0 = (int)(ii - (long long)i2 * N[0]);
        const int len = (int)(j1 - j0 + 1);
        seg[s] = make_int4(i0, i2, len, (int)cum);
        while (cur_plane <= i3) plane[cur_plane++] = s;
        cum += len;
    }
    while (cur_plane <= N[2]) plane[cur_plane++] = nseg;
    nvctr = (int)cum;
    return WVLH_OK;
}

static void region_free(wvlh_region *r)
{
    if (!r) return;
    if (r->mem) {
        cudaSetDevice(r->device);
        cudaFree(r->mem);
    }
    delete r;
}

// Validate, decode and upload the keys of one region (one device block).
static int region_make(int device, const wvlh_locreg &L, wvlh_region **out)
{
    *out = nullptr;
    for (int k = 0; k < 3; ++k) {
        if (L.n[k] < 1 || L.n[k] > 1024) return WVLH_ERR_ARG;
        // the periodic analysis/synthesis index arithmetic assumes at least 8 coarse cells
        if (L.periodic[k] && L.n[k] < 8) return WVLH_ERR_ARG;
    }
    if (L.nseg_c < 0 || L.nseg_f < 0) return WVLH_ERR_ARG;
    std::vector<int4> sc, sf;
    std::vector<int> pc, pf;
    int nvc = 0, nvf = 0, rc;
    if ((rc = decode_keys(L.n, L.nseg_c, L.keyg_c, L.keyv_c, sc, pc, nvc))) return rc;
    if ((rc = decode_keys(L.n, L.nseg_f, L.keyg_f, L.keyv_f, sf, pf, nvf))) return rc;
    wvlh_region *r = new wvlh_region();
    r->device = device;
    LrDev &d = r->lr;
    for (int k = 0; k < 3; ++k) {
        d.N[k] = L.n[k];
        d.per[k] = L.periodic[k] ? 1 : 0;
        d.hgrid[k] = L.hgrid[k];
        r->hgrid[k] = L.hgrid[k];
    }
    d.nseg_c = L.nseg_c;
    d.nseg_f = L.nseg_f;
    d.nvctr_c = nvc;
    d.nvctr_f = nvf;
    std::vector<uint32_t> kgc(L.keyg_c, L.keyg_c + 2 * (size_t)L.nseg_c), kvc(L.keyv_c, L.keyv_c + L.nseg_c);
    std::vector<uint32_t> kgf(L.keyg_f, L.keyg_f + 2 * (size_t)L.nseg_f), kvf(L.keyv_f, L.keyv_f + L.nseg_f);
    Packer pk;
    pk.add(sc, &d.seg_c);
    pk.add(sf, &d.seg_f);
    pk.add(pc, &d.plane_c);
    pk.add(pf, &d.plane_f);
    pk.add(kgc, &r->keyg_c);
    pk.add(kvc, &r->keyv_c);
    pk.add(kgf, &r->keyg_f);
    pk.add(kvf, &r->keyv_f);
    if (cudaMalloc(&r->mem, pk.img.size()) != cudaSuccess) {
        r->mem = nullptr;
        region_free(r);
        return WVLH_ERR_NOMEM;
    }
    if (cudaMemcpy(r->mem, pk.img.data(), pk.img.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        region_free(r);
        return WVLH_ERR_CUDA;
    }
    pk.place(r->mem);
    *out = r;
    return WVLH_OK;
}

extern "C" int wvlh_region_create(wvlh_ctx *ctx, const wvlh_locreg *lr, wvlh_region **out)
{
    if (!ctx || !lr || !out) return fail(WVLH_ERR_ARG);
    CK(cudaSetDevice(ctx->device));
    const int rc = region_make(ctx->device, *lr, out);
    return rc ? fail(rc) : WVLH_OK;
}

extern "C" int wvlh_region_destroy(wvlh_region *r)
{
    region_free(r);
    return WVLH_OK;
}

extern "C" int64_t wvlh_region_psi_size(const wvlh_region *r)
{
    return r ? r->lr.nvctr_c + 7LL * r->lr.nvctr_f : -1;
}

extern "C" int64_t wvlh_region_grid_size(const wvlh_region *r)
{
    if (!r) return -1;
    long long n = 1;
    for (int k = 0; k < 3; ++k) n *= isf_len(r->lr.N[k], r->lr.per[k]);
    return n;
}

// scratch elements of one orbital of a region in the fused kernels (P, Q, Z)
static long long orbital_scratch(const LrDev &d)
{
    const int G3 = 2 * d.N[2];
    const int F1 = fine_len(d.N[0], d.per[0]), F2 = fine_len(d.N[1], d.per[1]);
    const int I1 = isf_len(d.N[0], d.per[0]), I2 = isf_len(d.N[1], d.per[1]);
    return (long long)G3 * F2 * F1 * 2 + (long long)G3 * I2 * I1;
}

extern "C" int64_t wvlh_region_scratch_bytes(const wvlh_region *r, int precision)
{
    return r ? orbital_scratch(r->lr) * (precision == 32 ? 4 : 8) : -1;
}

// Lay out the orbitals of a batch over its regions (b->lr): scratch slices,
// fused-kernel work lists, energy partial slots, density groups and chunks.
// pot_key[o]: element offset of the orbital's potential (packed mode);
// den_key[o]: identity of its density grid (offset, or address in orbital
// mode); abs: per-orbital buffers (orbital mode) or null.
static void layout(wvlh_batch *b, const std::vector<int> &orb_lr, const std::vector<long long> &pot_key,
                   const std::vector<long long> &den_key, const wvlh_orbital *abs, Packer &pk)
{
    Plan &p = b->plan;
    const int nlr = (int)b->lr.size(), norb = (int)orb_lr.size();
    p.nlr = nlr;
    p.norb = norb;
    std::vector<LrDev> lrd(nlr);
    for (int l = 0; l < nlr; ++l) {
        lrd[l] = b->lr[l]->lr;
        for (int k = 0; k < 3; ++k) {
            p.lr_N.push_back(lrd[l].N[k]);
            p.lr_per.push_back(lrd[l].per[k]);
        }
    }
    std::vector<OrbDev> od(norb);
    std::vector<int> pre13(1, 0), pre2(1, 0), pre2p(1, 0), orb_len;
    std::vector<long long> orb_off;
    long long psi_off = 0, scr = 0;
    int stride = 0;
    size_t planeA = 0, planeB = 0, sm2_elems = 0;
    std::vector<PlaneShape> shapes32, shapes64;  // plane geometry per orbital (CTA-size choice)
    b->pot_off.assign(pot_key.begin(), pot_key.end());
    for (int o = 0; o < norb; ++o) {
        const int l = orb_lr[o];
        const LrDev &d = lrd[l];
        const int N1 = d.N[0], N2 = d.N[1], N3 = d.N[2];
        const int G3 = 2 * N3;
        const int F1 = fine_len(N1, d.per[0]), F2 = fine_len(N2, d.per[1]), F3 = fine_len(N3, d.per[2]);
        const int I1 = isf_len(N1, d.per[0]), I2 = isf_len(N2, d.per[1]), I3 = isf_len(N3, d.per[2]);
        OrbDev &q = od[o];
        q.lr = l;
        q.pad = 0;
        q.psi = psi_off;
        q.pot = pot_key[o];
        q.sP = scr;
        scr += (long long)G3 * F2 * F1;
        q.sQ = scr;
        scr += (long long)G3 * I2 * I1;
        q.sZ = scr;
        scr += (long long)G3 * F2 * F1;
        q.c = 0.0;
        q.in_ptr = abs ? abs[o].psi : nullptr;
        q.out_ptr = abs ? abs[o].hpsi : nullptr;
        q.pot_ptr = abs ? abs[o].pot : nullptr;
        p.orb_lr.push_back(l);
        p.orb_psi.push_back(psi_off);
        const int len = d.nvctr_c + 7 * d.nvctr_f;
        orb_off.push_back(psi_off);
        orb_len.push_back(len);
        psi_off += len;
        const int ntx0 = (I1 + TX_ - 1) / TX_, nty0 = (I2 + TY_ - 1) / TY_;
        const int ntx1 = (F1 + TX_ - 1) / TX_, nty1 = (F2 + TY_ - 1) / TY_;
        pre13.push_back(pre13.back() + G3);
        pre2.push_back(pre2.back() + ntx0 * nty0);
        pre2p.push_back(pre2p.back() + ntx1 * nty1);
        stride = std::max(stride, std::max(ntx0 * nty0, ntx1 * nty1 + G3));
        // plane buffer A: rows (y) x pitch (x); B holds P (F2 rows x pitch)
        // or a transposed plane (lines along x, each at the vec_pitch of its
        // y length).  Coarse lines are stored with the wavelet half at an
        // even offset (coarse_width).
        const int W1 = coarse_width(N1), W2 = coarse_width(N2);
        const int pitch = vec_pitch(std::max(W1, std::max(F1, I1)));
        const int rows = std::max(W2, std::max(F2, I2));
        const long long bT = std::max(std::max((long long)F1 * vec_pitch(W2), (long long)I1 * vec_pitch(F2)),
                                      std::max((long long)F1 * vec_pitch(I2), (long long)W1 * vec_pitch(F2)));
        const long long bsz = std::max((long long)F2 * pitch, bT);
        planeA = std::max(planeA, (size_t)rows * pitch);
        {
            const long long len = std::max(W1, std::max(F1, I1)), w = (long long)G3 * rows * pitch;
            const long long ab = (long long)rows * pitch + bsz;
            shapes32.push_back(PlaneShape{rows, len, ab * 4, w});
            shapes64.push_back(PlaneShape{rows, len, ab * 8, w});
        }
        planeB = std::max(planeB, (size_t)bsz);
        const int zl = std::max(G3, std::max(F3, I3));
        sm2_elems = std::max(sm2_elems, (size_t)2 * zl * TX_ * TY_);
    }
    p.psi_total = psi_off;
    p.all_periodic = true;
    for (int v : p.lr_per) p.all_periodic = p.all_periodic && v == 1;
    p.scratch_elems = (scr + 1) & ~1LL;  // even: the global plane slices after it start on a point pair
    {
        // one region for every orbital: regular (x, y, z, orbital) plane tensors
        bool one = norb > 0;
        for (int o = 1; o < norb && one; ++o) one = orb_lr[o] == orb_lr[0];
        if (one) {
            const LrDev &d = lrd[orb_lr[0]];
            const long long G3 = 2LL * d.N[2], F1 = fine_len(d.N[0], d.per[0]), F2 = fine_len(d.N[1], d.per[1]),
                            I1 = isf_len(d.N[0], d.per[0]), I2 = isf_len(d.N[1], d.per[1]);
            p.orb_scratch = 2 * G3 * F2 * F1 + G3 * I2 * I1;
            const long long dims[5] = {G3, F1, F2, I1, I2};
            for (int k = 0; k < 5; ++k) p.tile_dims[k] = dims[k];
        }
    }
    p.part_stride = stride;
    p.plane_threads[0] = choose_plane_threads(shapes32, true);
    p.plane_threads[1] = choose_plane_threads(shapes64, false);
    p.plane_threads_pre[0] = p.plane_threads[0];
    p.plane_threads_pre[1] = p.plane_threads[1];
    apply_tuned(p);   // a measured choice for this shape, when wvlh_batch_autotune made one
    p.plane_elems = (long long)planeA;
    p.planeB_elems = (long long)planeB;
    p.smem13[0] = (planeA + planeB) * sizeof(float);
    p.smem13[1] = (planeA + planeB) * sizeof(double);
    p.smem2[0] = sm2_elems * sizeof(float);
    p.smem2[1] = sm2_elems * sizeof(double);
    p.n_work13 = pre13.back();
    p.n_work2 = pre2.back();
    p.n_work2p = pre2p.back();
    // density: group the orbitals by density grid (same key, one region),
    // split each group in chunks of at most kDenChunk orbitals
    constexpr int kDenChunk = 32;
    std::vector<int> order(norb);
    for (int o = 0; o < norb; ++o) order[o] = o;
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) {
        return den_key[a] != den_key[c] ? den_key[a] < den_key[c] : orb_lr[a] < orb_lr[c];
    });
    std::vector<int> chunk_start, chunk_orbs, group_chunk_start, group_n;
    std::vector<long long> chunk_part, group_rho;
    std::vector<int> pred(1, 0);
    long long den = 0;
    b->density_ok = true;
    for (int i = 0; i < norb;) {
        int j = i;
        while (j < norb && den_key[order[j]] == den_key[order[i]]) {
            if (orb_lr[order[j]] != orb_lr[order[i]]) b->density_ok = false;  // one grid, one region
            ++j;
        }
        const LrDev &d = lrd[orb_lr[order[i]]];
        const int I1 = isf_len(d.N[0], d.per[0]), I2 = isf_len(d.N[1], d.per[1]), I3 = isf_len(d.N[2], d.per[2]);
        // accumulators of kd_density: 32 per thread, 48 for the larger grids
        if (I3 * TX_ * TY_ > 48 * kZThreads) b->density_ok = false;
        if (I3 * TX_ * TY_ > 32 * kZThreads) p.den_acc = 48;
        group_chunk_start.push_back((int)chunk_start.size());
        group_rho.push_back(den_key[order[i]]);
        group_n.push_back(I1 * I2 * I3);
        p.max_group_n = std::max(p.max_group_n, I1 * I2 * I3);
        // a group of many orbitals is split in up to 8 chunks (one partial
        // density each) so that its tiles fill the GPU
        const int n = j - i;
        const int nch = std::min(n, std::max(8, (n + kDenChunk - 1) / kDenChunk));
        const int per_chunk = (n + nch - 1) / nch;
        for (int k = i; k < j; k += per_chunk) {
            chunk_start.push_back((int)chunk_orbs.size());
            for (int m = k; m < std::min(j, k + per_chunk); ++m) chunk_orbs.push_back(order[m]);
            chunk_part.push_back(den);
            den += (long long)I1 * I2 * I3;
            pred.push_back(pred.back() + ((I1 + TX_ - 1) / TX_) * ((I2 + TY_ - 1) / TY_));
        }
        i = j;
    }
    chunk_start.push_back((int)chunk_orbs.size());
    group_chunk_start.push_back((int)chunk_part.size());
    p.nchunk = (int)chunk_part.size();
    p.ngroup = (int)group_rho.size();
    p.part_den_elems = den;
    p.n_workd = pred.back();
    pk.add(lrd, &p.d_lr);
    pk.add(od, &p.d_orb);
    pk.add(pre13, &p.d_pre13);
    pk.add(pre2, &p.d_pre2);
    pk.add(pre2p, &p.d_pre2p);
    pk.add(pred, &p.d_pred);
    pk.add(chunk_start, &p.d_chunk_orb_start);
    pk.add(chunk_orbs, &p.d_chunk_orbs);
    pk.add(chunk_part, &p.d_chunk_part);
    pk.add(group_chunk_start, &p.d_group_chunk_start);
    pk.add(group_rho, &p.d_group_rho);
    pk.add(group_n, &p.d_group_n);
    pk.add(orb_off, &p.d_orb_off);
    pk.add(orb_len, &p.d_orb_len);
}

extern "C" int wvlh_batch_create(wvlh_ctx *ctx, int nlr, const wvlh_locreg *lrs, int norb, const int32_t *orb_lr,
                                 const int64_t *pot_offset, wvlh_batch **out)
{
    if (!ctx || !lrs || nlr <= 0 || norb <= 0 || !orb_lr || !out) return fail(WVLH_ERR_ARG);
    for (int o = 0; o < norb; ++o)
        if (orb_lr[o] < 0 || orb_lr[o] >= nlr) return fail(WVLH_ERR_ARG);
    CK(cudaSetDevice(ctx->device));
    wvlh_batch *b = new wvlh_batch();
    b->ctx = ctx;
    for (int l = 0; l < nlr; ++l) {
        wvlh_region *r = nullptr;
        const int rc = region_make(ctx->device, lrs[l], &r);
        if (rc) {
            wvlh_batch_destroy(b);
            return fail(rc);
        }
        b->own_regions.push_back(r);
        b->lr.push_back(r);
    }
    std::vector<int> ol(orb_lr, orb_lr + norb);
    std::vector<long long> pk_pot(norb);
    for (int o = 0; o < norb; ++o) pk_pot[o] = pot_offset ? pot_offset[o] : 0;
    Packer pk;
    layout(b, ol, pk_pot, pk_pot, nullptr, pk);
    if (cudaMalloc(&b->mem, pk.img.size()) != cudaSuccess) {
        b->mem = nullptr;
        wvlh_batch_destroy(b);
        return fail(WVLH_ERR_NOMEM);
    }
    if (cudaMemcpy(b->mem, pk.img.data(), pk.img.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        wvlh_batch_destroy(b);
        return fail(WVLH_ERR_CUDA);
    }
    pk.place(b->mem);
    *out = b;
    return WVLH_OK;
}

extern "C" int wvlh_batch_create_orbitals(wvlh_ctx *ctx, int norb, const wvlh_orbital *orbs, wvlh_batch **out)
{
    if (!ctx || norb <= 0 || !orbs || !out) return fail(WVLH_ERR_ARG);
    std::map<const wvlh_region *, int> index;
    std::vector<int> ol(norb);
    std::vector<long long> pot(norb, 0), den(norb);
    bool locham = true, locden = true;
    for (int o = 0; o < norb; ++o) {
        const wvlh_orbital &q = orbs[o];
        if (!q.region || q.region->device != ctx->device || !q.psi) return fail(WVLH_ERR_ARG);
        auto it = index.find(q.region);
        ol[o] = it != index.end() ? it->second : (index[q.region] = (int)index.size());
        den[o] = (long long)(uintptr_t)q.rho;
        locham = locham && q.hpsi && q.pot;
        locden = locden && q.rho;
    }
    CK(cudaSetDevice(ctx->device));
    wvlh_batch *b = new wvlh_batch();
    b->ctx = ctx;
    b->orbital_mode = true;
    b->lr.resize(index.size());
    for (auto &kv : index) b->lr[kv.second] = kv.first;
    Packer pk;
    layout(b, ol, pot, den, orbs, pk);
    b->can_locham = locham;
    b->can_locden = locden && b->density_ok;
    // the tables replace the previous batch's in the context arena, in stream
    // order: launches queued before this call still read the old tables
    int rc = ctx->arena.ensure(pk.img.size());
    if (rc) {
        wvlh_batch_destroy(b);
        return fail(rc);
    }
    if (cudaMemcpyAsync(ctx->arena.p, pk.img.data(), pk.img.size(), cudaMemcpyHostToDevice, ctx->stream) !=
        cudaSuccess) {
        wvlh_batch_destroy(b);
        return fail(WVLH_ERR_CUDA);
    }
    pk.place(ctx->arena.p);
    b->arena_gen = ++ctx->arena_gen;
    *out = b;
    return WVLH_OK;
}

extern "C" int wvlh_batch_destroy(wvlh_batch *b)
{
    if (!b) return WVLH_OK;
    if (b->mem) {
        cudaSetDevice(b->ctx->device);
        cudaFree(b->mem);
    }
    for (wvlh_batch *q : b->chunks) wvlh_batch_destroy(q);
    for (wvlh_region *r : b->own_regions) region_free(r);
    delete b;
    return WVLH_OK;
}

extern "C" int64_t wvlh_batch_psi_size(const wvlh_batch *b) { return b ? b->plan.psi_total : -1; }
extern "C" int64_t wvlh_batch_psi_offset(const wvlh_batch *b, int orb)
{
    return (b && orb >= 0 && orb < b->plan.norb) ? b->plan.orb_psi[orb] : -1;
}
extern "C" int64_t wvlh_batch_scratch_bytes(const wvlh_batch *b, int precision)
{
    return b ? b->plan.scratch_elems * (precision == 32 ? 4 : 8) : -1;
}

// an orbital batch's tables stay valid until the next orbital batch of its context
static int batch_usable(const wvlh_batch *b)
{
    if (b->orbital_mode && b->arena_gen != b->ctx->arena_gen) return WVLH_ERR_STALE;
    return WVLH_OK;
}

// dynamic shared memory a block of the current device may ask for (its
// opt-in limit less 1 KB for the kernels' static arrays), 0 when the limit
// cannot be read
static size_t sm_limit()
{
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess || v <= 1024)
        return 0;
    return (size_t)v - 1024;
}

extern "C" int wvlh_locham_batched(wvlh_batch *b, int precision, const void *psi, const void *pot, void *hpsi,
                                   double *ekin, double *epot, int accumulate)
{
    if (!b || (precision != 32 && precision != 64)) return fail(WVLH_ERR_ARG);
    // orbital batches carry their buffers per orbital; packed batches need the bases
    if (b->orbital_mode ? !b->can_locham : (!psi || !pot || !hpsi)) return fail(WVLH_ERR_ARG);
    int rc;
    if ((rc = batch_usable(b))) return fail(rc);
    wvlh_ctx *c = b->ctx;
    CK(cudaSetDevice(c->device));
    const Plan &p = b->plan;
    const int fp = precision == 64;
    const size_t lim = sm_limit();
    if (!lim) return fail(WVLH_ERR_CUDA);
    if ((size_t)p.plane_elems * (fp ? 8 : 4) > lim || p.smem2[fp] > lim) return fail(WVLH_ERR_TOO_LARGE);
    if ((rc = c->scratch.ensure((p.scratch_elems + plane_tmp_elems(p, fp)) * (fp ? 8 : 4))) ||
        (rc = c->part_pot.ensure(sizeof(double) * (size_t)p.norb * p.part_stride)) ||
        (rc = c->part_kin.ensure(sizeof(double) * (size_t)p.norb * p.part_stride)))
        return fail(rc);
    cudaError_t e;
    cudaEvent_t *ev = c->timing ? c->ev : nullptr;
    if (fp)
        e = launch_locham<double, double>(p, (const double *)psi, (const double *)pot, (double *)hpsi,
                                          (double *)c->scratch.p, (double *)c->part_pot.p, (double *)c->part_kin.p,
                                          ekin, epot, accumulate, c->stream, ev);
    else
        e = launch_locham<float, float>(p, (const float *)psi, (const float *)pot, (float *)hpsi,
                                        (float *)c->scratch.p, (double *)c->part_pot.p, (double *)c->part_kin.p,
                                        ekin, epot, accumulate, c->stream, ev);
    CK(e);
    if (ev) {
        // the events of this call are read before the next call reuses them
        CK(cudaEventSynchronize(ev[4]));
        for (int k = 0; k < 4; ++k) {
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
            c->kernel_ms[k] += ms;
        }
        c->timed_calls++;
    }
    return WVLH_OK;
}

extern "C" int wvlh_ctx_enable_timing(wvlh_ctx *ctx, int on)
{
    if (!ctx) return fail(WVLH_ERR_ARG);
    CK(cudaSetDevice(ctx->device));
    if (on && !ctx->ev[0])
        for (auto &e : ctx->ev) CK(cudaEventCreate(&e));
    ctx->timing = on ? 1 : 0;
    for (auto &m : ctx->kernel_ms) m = 0.0;
    ctx->timed_calls = 0;
    return WVLH_OK;
}

extern "C" int wvlh_ctx_kernel_times(wvlh_ctx *ctx, double *ms4, long long *ncalls)
{
    if (!ctx || !ms4) return fail(WVLH_ERR_ARG);
    for (int k = 0; k < 4; ++k) ms4[k] = ctx->kernel_ms[k];
    if (ncalls) *ncalls = ctx->timed_calls;
    return WVLH_OK;
}

extern "C" int wvlh_measure_fma_peak(int precision, int iters, double *tflops)
{
    if (!tflops || (precision != 32 && precision != 64) || iters <= 0) return fail(WVLH_ERR_ARG);
    float ms = 0.f;
    double flops = 0.0;
    CK(fma_probe(precision, iters, &ms, &flops, 0));
    *tflops = flops / (ms * 1e-3) / 1e12;
    return WVLH_OK;
}

namespace wvlh {
template <class T>
cudaError_t launch_locden(const Plan &p, const T *psi, const double *hfac, double *rho, T *scratch, double *part,
                          cudaStream_t st);
template <class T>
cudaError_t launch_precond(const Plan &p, int ncong, const double *cprec, T *x, const T *b, T *r, T *dvec, T *ad,
                           T *scratch, double *scal, double *hist, cudaStream_t st);
}  // namespace wvlh

extern "C" int wvlh_locden_batched(wvlh_batch *b, int precision, const void *psi, const double *hfac, double *rho)
{
    if (!b || !hfac || (precision != 32 && precision != 64)) return fail(WVLH_ERR_ARG);
    if (b->orbital_mode ? !b->can_locden : (!psi || !rho)) return fail(WVLH_ERR_ARG);
    if (!b->density_ok) return fail(WVLH_ERR_UNSUPPORTED);
    int rc;
    if ((rc = batch_usable(b))) return fail(rc);
    if (b->orbital_mode) rho = nullptr;  // the groups hold the density addresses
    wvlh_ctx *c = b->ctx;
    CK(cudaSetDevice(c->device));
    const Plan &p = b->plan;
    const int fp = precision == 64;
    const size_t lim = sm_limit();
    if (!lim) return fail(WVLH_ERR_CUDA);
    if ((size_t)p.plane_elems * (fp ? 8 : 4) > lim || p.smem2[fp] > lim) return fail(WVLH_ERR_TOO_LARGE);
    if ((rc = c->scratch.ensure((p.scratch_elems + plane_tmp_elems(p, fp)) * (fp ? 8 : 4))) ||
        (rc = c->den_part.ensure(sizeof(double) * (size_t)p.part_den_elems)))
        return fail(rc);
    cudaError_t e = fp ? launch_locden<double>(p, (const double *)psi, hfac, rho, (double *)c->scratch.p,
                                               (double *)c->den_part.p, c->stream)
                       : launch_locden<float>(p, (const float *)psi, hfac, rho, (float *)c->scratch.p,
                                              (double *)c->den_part.p, c->stream);
    CK(e);
    return WVLH_OK;
}

extern "C" int wvlh_precond_batched(wvlh_batch *b, int precision, int ncong, const double *cprec, void *x,
                                    const void *rhs, double *hist)
{
    if (!b || !cprec || !x || !rhs || ncong < 0 || (precision != 32 && precision != 64)) return fail(WVLH_ERR_ARG);
    if (b->orbital_mode) return fail(WVLH_ERR_UNSUPPORTED);  // CG vectors are packed
    wvlh_ctx *c = b->ctx;
    CK(cudaSetDevice(c->device));
    const Plan &p = b->plan;
    const int fp = precision == 64;
    const size_t lim = sm_limit();
    if (!lim) return fail(WVLH_ERR_CUDA);
    if ((size_t)p.plane_elems * (fp ? 8 : 4) > lim || p.smem2[fp] > lim) return fail(WVLH_ERR_TOO_LARGE);
    const size_t es = fp ? 8 : 4;
    const size_t nv = (size_t)p.psi_total * es;
    int rc;
    if ((rc = c->scratch.ensure((p.scratch_elems + plane_tmp_elems(p, fp)) * es)) || (rc = c->cg_r.ensure(nv)) || (rc = c->cg_d.ensure(nv)) ||
        (rc = c->cg_ad.ensure(nv)) || (rc = c->cg_scal.ensure(sizeof(double) * (size_t)p.norb * (5 + 16 + p.part_stride))))
        return fail(rc);
    cudaError_t e =
        fp ? launch_precond<double>(p, ncong, cprec, (double *)x, (const double *)rhs, (double *)c->cg_r.p,
                                    (double *)c->cg_d.p, (double *)c->cg_ad.p, (double *)c->scratch.p,
                                    (double *)c->cg_scal.p, hist, c->stream)
           : launch_precond<float>(p, ncong, cprec, (float *)x, (const float *)rhs, (float *)c->cg_r.p,
                                   (float *)c->cg_d.p, (float *)c->cg_ad.p, (float *)c->scratch.p,
                                   (double *)c->cg_scal.p, hist, c->stream);
    CK(e);
    return WVLH_OK;
}

namespace wvlh {
size_t overlap_workspace_bytes(int norb, long long K, int nsm, bool two);
template <class TI>
cudaError_t launch_overlap(int norb, long long K, long long ld, const TI *psi, const TI *psib, double *S,
                           double *work, int nsm, cudaStream_t st);
}  // namespace wvlh

// S = psi psi^T, or L = psi hpsi^T when hpsi is given
static int overlap_entry(wvlh_ctx *c, int precision, int norb, int64_t K, int64_t ld, const void *psi,
                         const void *hpsi, double *S)
{
    if (!c || !psi || !S || norb <= 0 || K <= 0 || ld < K || (precision != 32 && precision != 64))
        return fail(WVLH_ERR_ARG);
    CK(cudaSetDevice(c->device));
    int nsm = 0;
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
    int rc;
    if ((rc = c->ov_work.ensure(overlap_workspace_bytes(norb, K, nsm, hpsi != nullptr)))) return fail(rc);
    cudaError_t e = precision == 64
                        ? launch_overlap<double>(norb, K, ld, (const double *)psi, (const double *)hpsi, S,
                                                 (double *)c->ov_work.p, nsm, c->stream)
                        : launch_overlap<float>(norb, K, ld, (const float *)psi, (const float *)hpsi, S,
                                                (double *)c->ov_work.p, nsm, c->stream);
    CK(e);
    return WVLH_OK;
}

extern "C" int wvlh_overlap(wvlh_ctx *c, int precision, int norb, int64_t K, int64_t ld, const void *psi, double *S)
{
    return overlap_entry(c, precision, norb, K, ld, psi, nullptr, S);
}

extern "C" int wvlh_subspace_matrix(wvlh_ctx *c, int precision, int norb, int64_t K, int64_t ld, const void *psi,
                                    const void *hpsi, double *L)
{
    if (!hpsi) return fail(WVLH_ERR_ARG);
    return overlap_entry(c, precision, norb, K, ld, psi, hpsi, L);
}

namespace wvlh {
cudaError_t launch_panel_apply(int norb, long long K, long long ld, const double *M, int lower, double alpha,
                               const double *psi, double beta, double *C, cudaStream_t st);
}  // namespace wvlh

extern "C" int wvlh_panel_apply(wvlh_ctx *c, int norb, int64_t K, int64_t ld, const double *M, int lower,
                                double alpha, const double *psi, double beta, double *out)
{
    if (!c || !M || !psi || !out || norb <= 0 || K <= 0 || ld < K || psi == out) return fail(WVLH_ERR_ARG);
    if (((uintptr_t)psi % 8) || ((uintptr_t)out % 8) || ((uintptr_t)M % 8)) return fail(WVLH_ERR_ARG);
    CK(cudaSetDevice(c->device));
    CK(launch_panel_apply(norb, K, ld, M, lower, alpha, psi, beta, out, c->stream));
    return WVLH_OK;
}

// ---------------------------------------------------------------------------
// Measured choice of the plane kernels' block size.  The analytic model of
// choose_plane_threads is a starting point; wvlh_batch_autotune times the
// batch's own local Hamiltonian with every candidate block size and keeps the
// fastest, both in the batch and in a process-wide table keyed by the batch's
// shape (operation, precision and every orbital's box), which later batches of
// the same shape read at creation.  wvlh_batch_autotune_precond does the same
// for the preconditioner operator, whose plane kernels run fewer passes per
// plane and so may prefer another size.
static std::mutex g_tune_mu;
static std::map<std::string, int> g_tuned;

// what: 0 plane kernels, 1 z kernel; pre: the preconditioner operator
static std::string tune_key(const Plan &p, int fp, bool pre = false, int what = 0)
{
    std::string k = std::string(what ? "z" : "") + (pre ? "p" : "") + (fp ? "64" : "32");
    for (int o = 0; o < p.norb; ++o) {
        const int l = p.orb_lr[o];
        char buf[64];
        snprintf(buf, sizeof buf, "|%d,%d,%d,%d%d%d", p.lr_N[3 * l], p.lr_N[3 * l + 1], p.lr_N[3 * l + 2],
                 p.lr_per[3 * l], p.lr_per[3 * l + 1], p.lr_per[3 * l + 2]);
        k += buf;
    }
    return k;
}

// the block sizes the plane kernels are compiled for
static const int kTune32[5] = {1024, 512, kPlaneThreads, 256, 128};
static const int kTune64[4] = {512, kPlaneThreads, 256, 128};
// the block sizes the FP32 z kernel is compiled for
static const int kTuneZ32[3] = {kZThreads, 320, 384};

static void apply_tuned(Plan &p)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (int fp = 0; fp < 2; ++fp) {
        auto it = g_tuned.find(tune_key(p, fp));
        if (it != g_tuned.end()) p.plane_threads[fp] = it->second;
        it = g_tuned.find(tune_key(p, fp, true));
        if (it != g_tuned.end()) p.plane_threads_pre[fp] = it->second;
        it = g_tuned.find(tune_key(p, fp, false, 1));
        if (it != g_tuned.end()) p.z_threads[fp] = it->second;
        it = g_tuned.find(tune_key(p, fp, true, 1));
        if (it != g_tuned.end()) p.z_threads_pre[fp] = it->second;
    }
}

// Times fn() (reps calls after one warm-up) with each candidate block size
// written into *slot; leaves the fastest in *slot and returns it in *chosen.
template <class F>
static int time_candidates(wvlh_ctx *c, int *slot, const int *cs, int n, int reps, F &&fn, int *chosen, int *cand,
                           double *ms, int *ncand)
{
    cudaEvent_t a, z;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&z));
    int best = *slot;
    double best_ms = -1.0;
    int rc = WVLH_OK;
    for (int k = 0; k < n && rc == WVLH_OK; ++k) {
        *slot = cs[k];
        rc = fn();   // warm-up
        cudaEventRecord(a, c->stream);
        for (int r = 0; r < reps && rc == WVLH_OK; ++r) rc = fn();
        cudaEventRecord(z, c->stream);
        if (rc) break;
        cudaEventSynchronize(z);
        float t = 0.f;
        cudaEventElapsedTime(&t, a, z);
        const double per = t / reps;
        if (cand) cand[k] = cs[k];
        if (ms) ms[k] = per;
        if (best_ms < 0 || per < best_ms) {
            best_ms = per;
            best = cs[k];
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(z);
    *slot = best;
    if (rc) return rc;
    if (chosen) *chosen = best;
    if (ncand) *ncand = n;
    return WVLH_OK;
}

extern "C" int wvlh_batch_autotune(wvlh_batch *b, int precision, const void *psi, const void *pot, void *hpsi,
                                   double *ekin, double *epot, int reps, int *chosen, int *cand, double *ms,
                                   int *ncand)
{
    if (!b || (precision != 32 && precision != 64) || reps < 1) return fail(WVLH_ERR_ARG);
    wvlh_ctx *c = b->ctx;
    CK(cudaSetDevice(c->device));
    const int fp = precision == 64;
    auto call = [&] { return wvlh_locham_batched(b, precision, psi, pot, hpsi, ekin, epot, 0); };
    int rc = time_candidates(c, &b->plan.plane_threads[fp], fp ? kTune64 : kTune32, fp ? 4 : 5, reps, call, chosen,
                             cand, ms, ncand);
    // then the z kernel's block size (FP32), with the plane kernels' pick
    if (!rc && !fp) rc = time_candidates(c, &b->plan.z_threads[0], kTuneZ32, 3, reps, call, nullptr, nullptr, nullptr, nullptr);
    if (rc) return fail(rc);
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned[tune_key(b->plan, fp)] = b->plan.plane_threads[fp];
    g_tuned[tune_key(b->plan, fp, false, 1)] = b->plan.z_threads[fp];
    return WVLH_OK;
}

extern "C" int wvlh_batch_block_sizes(const wvlh_batch *b, int *sizes)
{
    if (!b || !sizes) return fail(WVLH_ERR_ARG);
    const Plan &p = b->plan;
    const int v[8] = {p.plane_threads[0], p.plane_threads[1], p.z_threads[0], p.z_threads[1],
                      p.plane_threads_pre[0], p.plane_threads_pre[1], p.z_threads_pre[0], p.z_threads_pre[1]};
    for (int k = 0; k < 8; ++k) sizes[k] = v[k];
    return WVLH_OK;
}

extern "C" int wvlh_batch_autotune_precond(wvlh_batch *b, int precision, int ncong, const double *cprec, void *x,
                                           const void *rhs, int reps, int *chosen, int *cand, double *ms, int *ncand)
{
    if (!b || (precision != 32 && precision != 64) || reps < 1 || ncong < 0) return fail(WVLH_ERR_ARG);
    wvlh_ctx *c = b->ctx;
    CK(cudaSetDevice(c->device));
    const int fp = precision == 64;
    auto call = [&] { return wvlh_precond_batched(b, precision, ncong, cprec, x, rhs, nullptr); };
    int rc = time_candidates(c, &b->plan.plane_threads_pre[fp], fp ? kTune64 : kTune32, fp ? 4 : 5, reps, call,
                             chosen, cand, ms, ncand);
    if (!rc && !fp)
        rc = time_candidates(c, &b->plan.z_threads_pre[0], kTuneZ32, 3, reps, call, nullptr, nullptr, nullptr, nullptr);
    if (rc) return fail(rc);
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned[tune_key(b->plan, fp, true)] = b->plan.plane_threads_pre[fp];
    g_tuned[tune_key(b->plan, fp, true, 1)] = b->plan.z_threads_pre[fp];
    return WVLH_OK;
}

static long long pot_extent(const wvlh_batch *b)
{
    long long m = 0;
    for (int o = 0; o < b->plan.norb; ++o) {
        const int l = b->plan.orb_lr[o];
        long long n = 1;
        for (int k = 0; k < 3; ++k) n *= isf_len(b->plan.lr_N[3 * l + k], b->plan.lr_per[3 * l + k]);
        m = std::max(m, b->pot_off[o] + n);
    }
    return m;
}

// Sub-batch of the orbitals [o0, o1) of a packed batch: same regions and
// potential offsets, coefficients counted from the range's first orbital.
static int make_chunk(const wvlh_batch *parent, int o0, int o1, wvlh_batch **out)
{
    wvlh_batch *q = new wvlh_batch();
    q->ctx = parent->ctx;
    q->lr = parent->lr;
    std::vector<int> ol(parent->plan.orb_lr.begin() + o0, parent->plan.orb_lr.begin() + o1);
    std::vector<long long> pot(parent->pot_off.begin() + o0, parent->pot_off.begin() + o1);
    Packer pk;
    layout(q, ol, pot, pot, nullptr, pk);
    if (cudaMalloc(&q->mem, pk.img.size()) != cudaSuccess) {
        q->mem = nullptr;
        wvlh_batch_destroy(q);
        return WVLH_ERR_NOMEM;
    }
    if (cudaMemcpy(q->mem, pk.img.data(), pk.img.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        wvlh_batch_destroy(q);
        return WVLH_ERR_CUDA;
    }
    pk.place(q->mem);
    *out = q;
    return WVLH_OK;
}

// Host buffers: the orbitals go through in chunks that alternate between the
// context's stream and a second one, so that the upload of one chunk, the
// kernels of the previous one and the download of the one before overlap.
extern "C" int wvlh_locham_batched_host(wvlh_batch *b, int precision, const void *psi, const void *pot, void *hpsi,
                                        double *ekin, double *epot)
{
    if (!b || !psi || !pot || !hpsi || (precision != 32 && precision != 64)) return fail(WVLH_ERR_ARG);
    if (b->orbital_mode) return fail(WVLH_ERR_UNSUPPORTED);
    wvlh_ctx *c = b->ctx;
    CK(cudaSetDevice(c->device));
    const int fp = precision == 64;
    const size_t es = fp ? 8 : 4;
    const Plan &p = b->plan;
    const size_t npsi = (size_t)p.psi_total * es, npot = (size_t)pot_extent(b) * es;
    const size_t ne = sizeof(double) * p.norb;
    const size_t lim = sm_limit();
    if (!lim) return fail(WVLH_ERR_CUDA);
    if ((size_t)p.plane_elems * es > lim || p.smem2[fp] > lim) return fail(WVLH_ERR_TOO_LARGE);
    int rc;
    if ((rc = c->io_psi.ensure(npsi)) || (rc = c->io_hpsi.ensure(npsi)) || (rc = c->io_pot.ensure(npot)) ||
        (rc = c->io_e.ensure(2 * ne)))
        return fail(rc);
    // chunks of at least 8 orbitals, up to 32 (one chunk for small batches): the
    // first upload and the last download are the parts that nothing overlaps
    if (b->chunks.empty()) {
        const int nch = p.norb >= 16 ? std::min(32, p.norb / 8) : 1;
        const int per = (p.norb + nch - 1) / nch;
        for (int o0 = 0; o0 < p.norb; o0 += per) {
            wvlh_batch *q = nullptr;
            if ((rc = make_chunk(b, o0, std::min(p.norb, o0 + per), &q))) {
                for (wvlh_batch *x : b->chunks) wvlh_batch_destroy(x);
                b->chunks.clear();
                b->chunk_o0.clear();
                return fail(rc);
            }
            b->chunks.push_back(q);
            b->chunk_o0.push_back(o0);
        }
    }
    const size_t nch = b->chunks.size();
    if (!c->aux) CK(cudaStreamCreateWithFlags(&c->aux, cudaStreamNonBlocking));
    if (!c->aux2) CK(cudaStreamCreateWithFlags(&c->aux2, cudaStreamNonBlocking));
    if (!c->ev_a) CK(cudaEventCreateWithFlags(&c->ev_a, cudaEventDisableTiming));
    while (c->ev_in.size() < nch) {
        cudaEvent_t e1, e2;
        CK(cudaEventCreateWithFlags(&e1, cudaEventDisableTiming));
        c->ev_in.push_back(e1);
        CK(cudaEventCreateWithFlags(&e2, cudaEventDisableTiming));
        c->ev_cmp.push_back(e2);
    }
    // the chunks run one after another on the context's stream and share its scratch
    for (size_t k = 0; k < nch; ++k) {
        const Plan &q = b->chunks[k]->plan;
        if ((rc = c->scratch.ensure((q.scratch_elems + plane_tmp_elems(q, fp)) * es)) ||
            (rc = c->part_pot.ensure(sizeof(double) * (size_t)q.norb * q.part_stride)) ||
            (rc = c->part_kin.ensure(sizeof(double) * (size_t)q.norb * q.part_stride)))
            return fail(rc);
    }
    // three queues: uploads (aux) back to back, the chunk computations (the
    // context's stream) as their inputs arrive, downloads (aux2) as each chunk
    // is computed; both copy directions stay busy for the whole call
    cudaStream_t cs = c->stream, up = c->aux, down = c->aux2;
    unsigned char *dpsi = (unsigned char *)c->io_psi.p, *dh = (unsigned char *)c->io_hpsi.p;
    double *de = (double *)c->io_e.p;
    CK(cudaEventRecord(c->ev_a, cs));   // after earlier work on the context's stream
    CK(cudaStreamWaitEvent(up, c->ev_a, 0));
    CK(cudaStreamWaitEvent(down, c->ev_a, 0));
    CK(cudaMemcpyAsync(c->io_pot.p, pot, npot, cudaMemcpyHostToDevice, up));
    for (size_t k = 0; k < nch; ++k) {
        const size_t off = (size_t)p.orb_psi[b->chunk_o0[k]] * es, n = (size_t)b->chunks[k]->plan.psi_total * es;
        CK(cudaMemcpyAsync(dpsi + off, (const unsigned char *)psi + off, n, cudaMemcpyHostToDevice, up));
        CK(cudaEventRecord(c->ev_in[k], up));
    }
    for (size_t k = 0; k < nch; ++k) {
        const Plan &q = b->chunks[k]->plan;
        const int o0 = b->chunk_o0[k];
        const size_t off = (size_t)p.orb_psi[o0] * es;
        CK(cudaStreamWaitEvent(cs, c->ev_in[k], 0));
        cudaError_t e;
        if (fp)
            e = launch_locham<double, double>(q, (const double *)(dpsi + off), (const double *)c->io_pot.p,
                                              (double *)(dh + off), (double *)c->scratch.p, (double *)c->part_pot.p,
                                              (double *)c->part_kin.p, de + o0, de + p.norb + o0, 0, cs, nullptr);
        else
            e = launch_locham<float, float>(q, (const float *)(dpsi + off), (const float *)c->io_pot.p,
                                            (float *)(dh + off), (float *)c->scratch.p, (double *)c->part_pot.p,
                                            (double *)c->part_kin.p, de + o0, de + p.norb + o0, 0, cs, nullptr);
        CK(e);
        CK(cudaEventRecord(c->ev_cmp[k], cs));
    }
    for (size_t k = 0; k < nch; ++k) {
        const size_t off = (size_t)p.orb_psi[b->chunk_o0[k]] * es, n = (size_t)b->chunks[k]->plan.psi_total * es;
        CK(cudaStreamWaitEvent(down, c->ev_cmp[k], 0));
        CK(cudaMemcpyAsync((unsigned char *)hpsi + off, dh + off, n, cudaMemcpyDeviceToHost, down));
    }
    if (ekin) CK(cudaMemcpyAsync(ekin, de, ne, cudaMemcpyDeviceToHost, down));
    if (epot) CK(cudaMemcpyAsync(epot, de + p.norb, ne, cudaMemcpyDeviceToHost, down));
    // the download queue waited for every computation, which waited for every upload
    CK(cudaStreamSynchronize(down));
    return WVLH_OK;
}

// ---------------------------------------------------------------------------
// plain FP64 chain, one kernel per 1D pass, orbitals of a region batched
__global__ void k_gather_orbitals(const double *__restrict__ psi, const long long *__restrict__ offs, int n,
                                  double *__restrict__ out, int forward)
{
    const int o = blockIdx.y;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (forward) out[(size_t)o * n + i] = psi[offs[o] + i];
        else ((double *)psi)[offs[o] + i] = out[(size_t)o * n + i];
    }
}

__global__ void k_energy_parts(size_t n, const double *__restrict__ x, const double *__restrict__ y,
                               double *__restrict__ part)
{
    __shared__ double red[32];
    x += blockIdx.y * n;
    y += blockIdx.y * n;
    double e = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        e += x[i] * y[i];
    const double s = block_sum(e, red);
    if (threadIdx.x == 0) part[blockIdx.y * gridDim.x + blockIdx.x] = s;
}

__global__ void k_potential_batch(size_t n, const double *__restrict__ pot, double *__restrict__ psir,
                                  double *__restrict__ part)
{
    __shared__ double red[32];
    psir += blockIdx.y * n;
    double e = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double r = psir[i];
        const double w = pot[i] * r;
        e += w * r;
        psir[i] = w;
    }
    const double s = block_sum(e, red);
    if (threadIdx.x == 0) part[blockIdx.y * gridDim.x + blockIdx.x] = s;
}

__global__ void k_sum_rows(const double *__restrict__ part, int ncol, int nrow, const long long *__restrict__ idx,
                           double *__restrict__ out, const double *__restrict__ sub)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrow) return;
    double s = 0.0;
    for (int i = 0; i < ncol; ++i) s += part[(size_t)r * ncol + i];
    const long long o = idx[r];
    out[o] = s - (sub ? sub[o] : 0.0);
}

extern "C" int wvlh_locham_plain_batched(wvlh_batch *b, const double *psi, const double *pot, double *hpsi,
                                         double *ekin, double *epot)
{
    if (!b || !psi || !pot || !hpsi || !ekin || !epot) return fail(WVLH_ERR_ARG);
    if (b->orbital_mode) return fail(WVLH_ERR_UNSUPPORTED);
    wvlh_ctx *c = b->ctx;
    CK(cudaSetDevice(c->device));
    cudaStream_t st = c->stream;
    const Plan &p = b->plan;
    constexpr int NPART = 64;
    for (int l = 0; l < p.nlr; ++l) {
        std::vector<long long> orbs, poffs;
        std::vector<long long> oidx;
        for (int o = 0; o < p.norb; ++o)
            if (p.orb_lr[o] == l) {
                orbs.push_back(p.orb_psi[o]);
                oidx.push_back(o);
            }
        if (orbs.empty()) continue;
        const int nb = (int)orbs.size();
        const int N1 = p.lr_N[3 * l], N2 = p.lr_N[3 * l + 1], N3 = p.lr_N[3 * l + 2];
        const int q1 = p.lr_per[3 * l], q2 = p.lr_per[3 * l + 1], q3 = p.lr_per[3 * l + 2];
        const int F1 = fine_len(N1, q1), F2 = fine_len(N2, q2), F3 = fine_len(N3, q3);
        const int I1 = isf_len(N1, q1), I2 = isf_len(N2, q2), I3 = isf_len(N3, q3);
        const size_t ni = (size_t)I1 * I2 * I3;
        const wvlh_region &R = *b->lr[l];
        const int nvc = R.lr.nvctr_c, nvf = R.lr.nvctr_f;
        const int ncomp = nvc + 7 * nvf;
        int rc;
        for (int k = 0; k < 4; ++k)
            if ((rc = c->plain[k].ensure(sizeof(double) * ni * nb))) return fail(rc);
        const size_t need = sizeof(double) * ((size_t)2 * nb * NPART + 2 * nb) + sizeof(long long) * 2 * nb;
        if ((rc = c->dotpart.ensure(need))) return fail(rc);
        double *W0 = (double *)c->plain[0].p, *W1 = (double *)c->plain[1].p, *W2 = (double *)c->plain[2].p,
               *W3 = (double *)c->plain[3].p;
        double *ppart = (double *)c->dotpart.p, *kpart = ppart + (size_t)nb * NPART;
        long long *d_offs = (long long *)(kpart + (size_t)nb * NPART);
        long long *d_oidx = d_offs + nb;
        CK(cudaMemcpyAsync(d_offs, orbs.data(), sizeof(long long) * nb, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(d_oidx, oidx.data(), sizeof(long long) * nb, cudaMemcpyHostToDevice, st));
        // W3 <- compressed psi of the region's orbitals, [c | f] contiguous per orbital
        k_gather_orbitals<<<dim3(64, nb), 256, 0, st>>>(psi, d_offs, ncomp, W3, 1);
        const int dims[3] = {N1, N2, N3};
        // uncompress (OpenCL/Uncompress.c:596-606): W3 -> W0
        CK(plain_uncompress(0, dims, R.lr.nseg_c, nvc, R.keyg_c, R.keyv_c, R.lr.nseg_f, nvf, R.keyg_f,
                            R.keyv_f, W3, W3 + nvc, W0, nullptr, nb, ncomp, ncomp, ni, st));
        // syn z, y, x (OpenCL/Wavelet.c:282-315): W0 -> W1 -> W0 -> W1 (X)
        CK(plain_syn1d(N3, 4 * N1 * N2, q3, W0, W1, nb, ni, ni, st));
        CK(plain_syn1d(N2, 2 * N1 * F3, q2, W1, W0, nb, ni, ni, st));
        CK(plain_syn1d(N1, F3 * F2, q1, W0, W1, nb, ni, ni, st));
        // MF z, y, x: W1 -> W0 -> W2 -> W0 (R)
        CK(plain_mf1d(q3 ? 0 : 2, F3, F1 * F2, W1, W0, nb, ni, ni, st));
        CK(plain_mf1d(q2 ? 0 : 2, F2, F1 * I3, W0, W2, nb, ni, ni, st));
        CK(plain_mf1d(q1 ? 0 : 2, F1, I3 * I2, W2, W0, nb, ni, ni, st));
        // V . R, epot (MagicFilter.c:327 potential_application)
        k_potential_batch<<<dim3(NPART, nb), 256, 0, st>>>(ni, pot + b->pot_off[oidx[0]], W0, ppart);
        // MF^T z, y, x: W0 -> W2 -> W0 -> W2 (Y0)
        CK(plain_mf1d(q3 ? 1 : 3, F3, I1 * I2, W0, W2, nb, ni, ni, st));
        CK(plain_mf1d(q2 ? 1 : 3, F2, I1 * F3, W2, W0, nb, ni, ni, st));
        CK(plain_mf1d(q1 ? 1 : 3, F1, F3 * F2, W0, W2, nb, ni, ni, st));
        // kinetic z, y, x (Kinetic.c:240-270): (x=W1, y=W2) -> (W0, W3) -> (W1, W2) -> (W0, W3)
        const double h1 = 0.5 * R.hgrid[0], h2 = 0.5 * R.hgrid[1], h3 = 0.5 * R.hgrid[2];
        CK(plain_kin1d(F3, F1 * F2, q3, -0.5 / (h3 * h3), W1, W0, W2, W3, nb, ni, ni, st));
        CK(plain_kin1d(F2, F1 * F3, q2, -0.5 / (h2 * h2), W0, W1, W3, W2, nb, ni, ni, st));
        CK(plain_kin1d(F1, F3 * F2, q1, -0.5 / (h1 * h1), W1, W0, W2, W3, nb, ni, ni, st));
        // <X|Y> = ekin + epot (Hamiltonian.c:60-62 dot_d_async)
        k_energy_parts<<<dim3(NPART, nb), 256, 0, st>>>((size_t)F1 * F2 * F3, W0, W3, kpart);
        // ana z, y, x: W3 -> W1 -> W3 -> W1
        CK(plain_ana1d(N3, F1 * F2, q3, W3, W1, nb, ni, ni, st));
        CK(plain_ana1d(N2, F1 * 2 * N3, q2, W1, W3, nb, ni, ni, st));
        CK(plain_ana1d(N1, 4 * N3 * N2, q1, W3, W1, nb, ni, ni, st));
        // compress (Uncompress.c:608-613): W1 -> W2 (compressed), scatter to hpsi
        CK(plain_uncompress(1, dims, R.lr.nseg_c, nvc, R.keyg_c, R.keyv_c, R.lr.nseg_f, nvf, R.keyg_f,
                            R.keyv_f, W2, W2 + nvc, W1, nullptr, nb, ncomp, ncomp, ni, st));
        k_gather_orbitals<<<dim3(64, nb), 256, 0, st>>>(hpsi, d_offs, ncomp, W2, 0);
        k_sum_rows<<<(nb + 127) / 128, 128, 0, st>>>(ppart, NPART, nb, d_oidx, epot, nullptr);
        k_sum_rows<<<(nb + 127) / 128, 128, 0, st>>>(kpart, NPART, nb, d_oidx, ekin, epot);
        CK(cudaGetLastError());
    }
    return WVLH_OK;
}

extern "C" void *wvlh_host_alloc(size_t bytes)
{
    void *p = nullptr;
    if (cudaMallocHost(&p, bytes) != cudaSuccess) return nullptr;
    return p;
}
extern "C" void wvlh_host_free(void *p)
{
    if (p) cudaFreeHost(p);
}

namespace wvlh {
template <class T>
cudaError_t launch_wpdot(int nseg_ac, const uint32_t *kg_ac, const uint32_t *kv_ac, int nseg_af,
                         const uint32_t *kg_af, const uint32_t *kv_af, int nvc_a, int nseg_bc, const uint32_t *kg_bc,
                         const uint32_t *kv_bc, int nseg_bf, const uint32_t *kg_bf, const uint32_t *kv_bf, int nvc_b,
                         int na, const T *a, long long lda, int nb, const T *b, long long ldb, double *out,
                         int4 *runs, cudaStream_t st);
}  // namespace wvlh

extern "C" int wvlh_wpdot(wvlh_ctx *c, int precision, const wvlh_region *ra, int na, const void *a, int64_t lda,
                          const wvlh_region *rb, int nb, const void *b, int64_t ldb, double *out)
{
    if (!c || !ra || !rb || !a || !b || !out || na <= 0 || nb <= 0 || (precision != 32 && precision != 64))
        return fail(WVLH_ERR_ARG);
    if (ra->device != c->device || rb->device != c->device) return fail(WVLH_ERR_ARG);
    for (int k = 0; k < 3; ++k)
        if (ra->lr.N[k] != rb->lr.N[k]) return fail(WVLH_ERR_ARG);  // keys of one box
    if (lda < wvlh_region_psi_size(ra) || ldb < wvlh_region_psi_size(rb) || na > 65535) return fail(WVLH_ERR_ARG);
    CK(cudaSetDevice(c->device));
    const int nrun = rb->lr.nseg_c + rb->lr.nseg_f;
    int rc;
    if ((rc = c->wp_runs.ensure(sizeof(int4) * (size_t)(nrun > 0 ? nrun : 1)))) return fail(rc);
    int4 *runs = (int4 *)c->wp_runs.p;
    cudaError_t e;
    if (precision == 64)
        e = launch_wpdot<double>(ra->lr.nseg_c, ra->keyg_c, ra->keyv_c, ra->lr.nseg_f, ra->keyg_f, ra->keyv_f,
                                 ra->lr.nvctr_c, rb->lr.nseg_c, rb->keyg_c, rb->keyv_c, rb->lr.nseg_f, rb->keyg_f,
                                 rb->keyv_f, rb->lr.nvctr_c, na, (const double *)a, lda, nb, (const double *)b, ldb,
                                 out, runs, c->stream);
    else
        e = launch_wpdot<float>(ra->lr.nseg_c, ra->keyg_c, ra->keyv_c, ra->lr.nseg_f, ra->keyg_f, ra->keyv_f,
                                ra->lr.nvctr_c, rb->lr.nseg_c, rb->keyg_c, rb->keyv_c, rb->lr.nseg_f, rb->keyg_f,
                                rb->keyv_f, rb->lr.nvctr_c, na, (const float *)a, lda, nb, (const float *)b, ldb, out,
                                runs, c->stream);
    CK(e);
    return WVLH_OK;
}

// ---------------------------------------------------------------------------
// CUDA graph of one packed-batch locham call (the same batch applied at every
// SCF iteration): the memsets and kernels are captured once and replayed with
// one launch.  The graph owns its scratch, so that later calls on the context
// (which may grow the context's buffers) cannot move memory under it.
struct wvlh_graph {
    wvlh_ctx *ctx = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    DevBuf scratch, part_pot, part_kin;
};

extern "C" int wvlh_graph_destroy(wvlh_graph *g)
{
    if (!g) return WVLH_OK;
    cudaSetDevice(g->ctx->device);
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    cudaDeviceSynchronize();
    g->scratch.release();
    g->part_pot.release();
    g->part_kin.release();
    delete g;
    return WVLH_OK;
}

extern "C" int wvlh_locham_graph_create(wvlh_batch *b, int precision, const void *psi, const void *pot, void *hpsi,
                                        double *ekin, double *epot, int accumulate, wvlh_graph **out)
{
    if (!b || !out || !psi || !pot || !hpsi || (precision != 32 && precision != 64)) return fail(WVLH_ERR_ARG);
    if (b->orbital_mode) return fail(WVLH_ERR_UNSUPPORTED);  // its tables live in a shared arena
    wvlh_ctx *c = b->ctx;
    CK(cudaSetDevice(c->device));
    const Plan &p = b->plan;
    const int fp = precision == 64;
    const size_t lim = sm_limit();
    if (!lim) return fail(WVLH_ERR_CUDA);
    if ((size_t)p.plane_elems * (fp ? 8 : 4) > lim || p.smem2[fp] > lim) return fail(WVLH_ERR_TOO_LARGE);
    wvlh_graph *g = new wvlh_graph();
    g->ctx = c;
    int rc;
    if ((rc = g->scratch.ensure((p.scratch_elems + plane_tmp_elems(p, fp)) * (fp ? 8 : 4))) ||
        (rc = g->part_pot.ensure(sizeof(double) * (size_t)p.norb * p.part_stride)) ||
        (rc = g->part_kin.ensure(sizeof(double) * (size_t)p.norb * p.part_stride))) {
        wvlh_graph_destroy(g);
        return fail(rc);
    }
    cudaStream_t cs = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        cudaError_t le;
        if (fp)
            le = launch_locham<double, double>(p, (const double *)psi, (const double *)pot, (double *)hpsi,
                                               (double *)g->scratch.p, (double *)g->part_pot.p,
                                               (double *)g->part_kin.p, ekin, epot, accumulate, cs, nullptr);
        else
            le = launch_locham<float, float>(p, (const float *)psi, (const float *)pot, (float *)hpsi,
                                             (float *)g->scratch.p, (double *)g->part_pot.p,
                                             (double *)g->part_kin.p, ekin, epot, accumulate, cs, nullptr);
        e = cudaStreamEndCapture(cs, &g->graph);
        if (le != cudaSuccess) e = le;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
    if (cs) cudaStreamDestroy(cs);
    if (e != cudaSuccess) {
        fprintf(stderr, "wvlh: %s\n", cudaGetErrorString(e));
        wvlh_graph_destroy(g);
        return fail(WVLH_ERR_CUDA);
    }
    *out = g;
    return WVLH_OK;
}

extern "C" int wvlh_graph_launch(wvlh_graph *g)
{
    if (!g) return fail(WVLH_ERR_ARG);
    CK(cudaSetDevice(g->ctx->device));
    CK(cudaGraphLaunch(g->exec, g->ctx->stream));
    return WVLH_OK;
}
