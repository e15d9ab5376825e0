// Batched ABI: contexts, batch plans (key validation and decoding, work
// tables) and the batched local-Hamiltonian entry points.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/wvlh.h"
#include "wvlh_common.cuh"
#include "wvlh_internal.h"
#include "wvlh_plain.h"

namespace wvlh {
template <class T, class TIO>
cudaError_t launch_locham(const Plan &p, const TIO *psi, const TIO *pot, TIO *hpsi, T *scratch, double *part_pot,
                          double *part_kin, double *ekin, double *epot, int accumulate, cudaStream_t st,
                          cudaEvent_t *ev);
cudaError_t fma_probe(int precision, int iters, float *ms, double *flops, cudaStream_t st);
void set_last_error(int code);
}  // namespace wvlh

using namespace wvlh;

// grow-only device buffer
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    int ensure(size_t b)
    {
        if (b <= bytes) return WVLH_OK;
        if (p) cudaFree(p);
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

struct wvlh_ctx {
    int device = 0;
    cudaStream_t stream = 0;
    DevBuf cg_r, cg_d, cg_ad, cg_scal, den_part, ov_work;
    // optional per-kernel timing of the fused locham (K1, K2, K3, reduction)
    int timing = 0;
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    double kernel_ms[4] = {0, 0, 0, 0};
    long long timed_calls = 0;
    DevBuf scratch, part_pot, part_kin, io_psi, io_pot, io_hpsi, io_e, plain[4], dotpart;
};

struct wvlh_batch {
    wvlh_ctx *ctx = nullptr;
    Plan plan;
    std::vector<int64_t> pot_off;
    bool density_ok = true;  // orbitals sharing a density grid share its region
    // raw 1-based keys per region on the device (plain path)
    std::vector<uint32_t *> d_keyg_c, d_keyv_c, d_keyg_f, d_keyv_f;
    std::vector<int> nvc, nvf, nsc, nsf;
    std::vector<double> hgrid;  // 3*nlr
};

static int fail(int code)
{
    set_last_error(code);
    return code;
}

#define CK(x)                                                  \
    do {                                                       \
        cudaError_t e_ = (x);                                  \
        if (e_ != cudaSuccess) {                               \
            fprintf(stderr, "wvlh: %s\n", cudaGetErrorString(e_)); \
            return fail(WVLH_ERR_CUDA);                        \
        }                                                      \
    } while (0)

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
    ctx->scratch.release();
    ctx->part_pot.release();
    ctx->part_kin.release();
    ctx->io_psi.release();
    ctx->io_pot.release();
    ctx->io_hpsi.release();
    ctx->io_e.release();
    for (auto &b : ctx->plain) b.release();
    ctx->dotpart.release();
    ctx->cg_r.release();
    ctx->cg_d.release();
    ctx->cg_ad.release();
    ctx->cg_scal.release();
    ctx->den_part.release();
    ctx->ov_work.release();
    for (auto &e : ctx->ev)
        if (e) cudaEventDestroy(e);
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

// Validate the reference's 1-based keys of one region and decode them into
// {i0, i2, len, jj0} plus per-plane segment ranges (wavelib/un-compress.f90:896-905).
static int decode_keys(const int *N, int nseg, const int32_t *keyg, const int32_t *keyv, std::vector<int4> &seg,
                       std::vector<int> &plane, int &nvctr)
{
    const long long n12 = (long long)N[0] * N[1], ntot = n12 * N[2];
    seg.resize(nseg);
    plane.assign(N[2] + 1, nseg);
    long long prev_end = 0;
    long long cum = 0;
    int cur_plane = 0;
    for (int s = 0; s < nseg; ++s) {
        const long long j0 = keyg[2 * s], j1 = keyg[2 * s + 1];
        if (j0 < 1 || j1 < j0 || j1 > ntot || j0 <= prev_end) return WVLH_ERR_KEYS;
        if ((j0 - 1) / N[0] != (j1 - 1) / N[0]) return WVLH_ERR_KEYS;  // segments stay on one x-line
        if ((long long)keyv[s] != cum + 1) return WVLH_ERR_KEYS;
        long long ii = j0 - 1;
        const int i3 = (int)(ii / n12);
        ii -= (long long)i3 * n12;
        const int i2 = (int)(ii / N[0]);
        const int i0 = (int)(ii - (long long)i2 * N[0]);
        const int len = (int)(j1 - j0 + 1);
        seg[s] = make_int4(i0, i2, len, (int)cum);
        while (cur_plane <= i3) plane[cur_plane++] = s;
        cum += len;
        prev_end = j1;
    }
    while (cur_plane <= N[2]) plane[cur_plane++] = nseg;
    nvctr = (int)cum;
    return WVLH_OK;
}

template <class T>
static int upload(Plan &p, const std::vector<T> &v, T **dst)
{
    *dst = nullptr;
    if (v.empty()) return WVLH_OK;
    if (cudaMalloc(dst, v.size() * sizeof(T)) != cudaSuccess) return WVLH_ERR_NOMEM;
    p.owned.push_back(*dst);
    if (cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) return WVLH_ERR_CUDA;
    return WVLH_OK;
}

extern "C" int wvlh_batch_create(wvlh_ctx *ctx, int nlr, const wvlh_locreg *lrs, int norb, const int32_t *orb_lr,
                                 const int64_t *pot_offset, wvlh_batch **out)
{
    if (!ctx || !lrs || nlr <= 0 || norb <= 0 || !orb_lr || !out) return fail(WVLH_ERR_ARG);
    CK(cudaSetDevice(ctx->device));
    wvlh_batch *b = new wvlh_batch();
    b->ctx = ctx;
    Plan &p = b->plan;
    p.nlr = nlr;
    p.norb = norb;
    std::vector<LrDev> lrd(nlr);
    b->hgrid.resize(3 * nlr);
    int rc = WVLH_OK;
    for (int l = 0; l < nlr && rc == WVLH_OK; ++l) {
        const wvlh_locreg &L = lrs[l];
        LrDev &d = lrd[l];
        for (int k = 0; k < 3; ++k) {
            if (L.n[k] < 1 || L.n[k] > 1024) rc = WVLH_ERR_ARG;
            // the periodic analysis/synthesis index arithmetic assumes at least 8 coarse cells
            if (L.periodic[k] && L.n[k] < 8) rc = WVLH_ERR_ARG;
            d.N[k] = L.n[k];
            d.per[k] = L.periodic[k] ? 1 : 0;
            d.hgrid[k] = L.hgrid[k];
            b->hgrid[3 * l + k] = L.hgrid[k];
            p.lr_N.push_back(L.n[k]);
            p.lr_per.push_back(d.per[k]);
        }
        if (rc) break;
        std::vector<int4> sc, sf;
        std::vector<int> pc, pf;
        int nvc = 0, nvf = 0;
        if (L.nseg_c < 0 || L.nseg_f < 0) rc = WVLH_ERR_ARG;
        if (!rc) rc = decode_keys(L.n, L.nseg_c, L.keyg_c, L.keyv_c, sc, pc, nvc);
        if (!rc) rc = decode_keys(L.n, L.nseg_f, L.keyg_f, L.keyv_f, sf, pf, nvf);
        if (rc) break;
        d.nseg_c = L.nseg_c;
        d.nseg_f = L.nseg_f;
        d.nvctr_c = nvc;
        d.nvctr_f = nvf;
        int4 *dsc, *dsf;
        int *dpc, *dpf;
        if ((rc = upload(p, sc, &dsc)) || (rc = upload(p, sf, &dsf)) || (rc = upload(p, pc, &dpc)) ||
            (rc = upload(p, pf, &dpf)))
            break;
        d.seg_c = dsc;
        d.seg_f = dsf;
        d.plane_c = dpc;
        d.plane_f = dpf;
        // raw keys for the plain path
        std::vector<uint32_t> kgc(2 * (size_t)L.nseg_c), kvc(L.nseg_c), kgf(2 * (size_t)L.nseg_f), kvf(L.nseg_f);
        for (int s = 0; s < 2 * L.nseg_c; ++s) kgc[s] = (uint32_t)L.keyg_c[s];
        for (int s = 0; s < L.nseg_c; ++s) kvc[s] = (uint32_t)L.keyv_c[s];
        for (int s = 0; s < 2 * L.nseg_f; ++s) kgf[s] = (uint32_t)L.keyg_f[s];
        for (int s = 0; s < L.nseg_f; ++s) kvf[s] = (uint32_t)L.keyv_f[s];
        uint32_t *a, *bb, *c, *dd;
        if ((rc = upload(p, kgc, &a)) || (rc = upload(p, kvc, &bb)) || (rc = upload(p, kgf, &c)) ||
            (rc = upload(p, kvf, &dd)))
            break;
        b->d_keyg_c.push_back(a);
        b->d_keyv_c.push_back(bb);
        b->d_keyg_f.push_back(c);
        b->d_keyv_f.push_back(dd);
        b->nvc.push_back(nvc);
        b->nvf.push_back(nvf);
        b->nsc.push_back(L.nseg_c);
        b->nsf.push_back(L.nseg_f);
    }
    if (rc) {
        wvlh_batch_destroy(b);
        return fail(rc);
    }
    // orbitals, scratch layout, work tables
    std::vector<OrbDev> od(norb);
    std::vector<int2> w13;
    std::vector<int> s13;
    std::vector<int4> w2, w2p;
    std::vector<int> s2, s2p, orb_len;
    std::vector<long long> orb_off;
    long long psi_off = 0, scr = 0;
    int stride = 0;
    size_t sm13_elems = 0, sm2_elems = 0;
    b->pot_off.resize(norb);
    for (int o = 0; o < norb; ++o) {
        const int l = orb_lr[o];
        if (l < 0 || l >= nlr) {
            wvlh_batch_destroy(b);
            return fail(WVLH_ERR_ARG);
        }
        const LrDev &d = lrd[l];
        const int N1 = d.N[0], N2 = d.N[1], N3 = d.N[2];
        const int G1 = 2 * N1, G2 = 2 * N2, G3 = 2 * N3;
        const int F1 = fine_len(N1, d.per[0]), F2 = fine_len(N2, d.per[1]), F3 = fine_len(N3, d.per[2]);
        const int I1 = isf_len(N1, d.per[0]), I2 = isf_len(N2, d.per[1]), I3 = isf_len(N3, d.per[2]);
        OrbDev &q = od[o];
        q.lr = l;
        q.psi = psi_off;
        q.pot = pot_offset ? pot_offset[o] : 0;
        b->pot_off[o] = q.pot;
        q.sP = scr;
        scr += (long long)G3 * F2 * F1;
        q.sQ = scr;
        scr += (long long)G3 * I2 * I1;
        q.sZ = scr;
        scr += (long long)G3 * F2 * F1;
        q.c = 0.0;
        p.orb_lr.push_back(l);
        p.orb_psi.push_back(psi_off);
        psi_off += d.nvctr_c + 7LL * d.nvctr_f;
        const int ntx0 = (I1 + TX_ - 1) / TX_, nty0 = (I2 + TY_ - 1) / TY_;
        const int ntx1 = (F1 + TX_ - 1) / TX_, nty1 = (F2 + TY_ - 1) / TY_;
        for (int ty = 0; ty < nty0; ++ty)
            for (int tx = 0; tx < ntx0; ++tx) {
                w2.push_back(make_int4(o, 0, tx * TX_, ty * TY_));
                s2.push_back(ty * ntx0 + tx);
            }
        for (int ty = 0; ty < nty1; ++ty)
            for (int tx = 0; tx < ntx1; ++tx) {
                w2.push_back(make_int4(o, 1, tx * TX_, ty * TY_));
                s2.push_back(ty * ntx1 + tx);
                w2p.push_back(make_int4(o, 1, tx * TX_, ty * TY_));
                s2p.push_back(ty * ntx1 + tx);
            }
        orb_off.push_back(psi_off - (d.nvctr_c + 7LL * d.nvctr_f));
        orb_len.push_back(d.nvctr_c + 7 * d.nvctr_f);
        for (int kz = 0; kz < G3; ++kz) {
            w13.push_back(make_int2(o, kz));
            s13.push_back(ntx1 * nty1 + kz);
        }
        stride = std::max(stride, std::max(ntx0 * nty0, ntx1 * nty1 + G3));
        const int pitch = std::max(G1, std::max(F1, I1)) | 1;
        const int rows = std::max(G2, std::max(F2, I2));
        sm13_elems = std::max(sm13_elems, (size_t)2 * rows * pitch);
        const int zl = std::max(G3, std::max(F3, I3));
        sm2_elems = std::max(sm2_elems, (size_t)2 * zl * TX_ * TY_);
    }
    p.psi_total = psi_off;
    p.all_periodic = true;
    for (int v : p.lr_per) p.all_periodic = p.all_periodic && v == 1;
    p.scratch_elems = scr;
    p.part_stride = stride;
    p.smem13[0] = sm13_elems * sizeof(float);
    p.smem13[1] = sm13_elems * sizeof(double);
    p.smem2[0] = sm2_elems * sizeof(float);
    p.smem2[1] = sm2_elems * sizeof(double);
    p.n_work13 = (int)w13.size();
    p.n_work2 = (int)w2.size();
    p.n_work2p = (int)w2p.size();
    // density: group the orbitals by density grid (same region and offset),
    // split each group in chunks of at most kDenChunk orbitals
    constexpr int kDenChunk = 32;
    std::vector<int> order(norb);
    for (int o = 0; o < norb; ++o) order[o] = o;
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) {
        return b->pot_off[a] != b->pot_off[c] ? b->pot_off[a] < b->pot_off[c] : orb_lr[a] < orb_lr[c];
    });
    std::vector<int> chunk_start, chunk_orbs, group_chunk_start, group_n;
    std::vector<long long> chunk_part, group_rho;
    std::vector<int4> wd;
    long long den = 0;
    b->density_ok = true;
    for (int i = 0; i < norb;) {
        int j = i;
        while (j < norb && b->pot_off[order[j]] == b->pot_off[order[i]]) {
            if (orb_lr[order[j]] != orb_lr[order[i]]) b->density_ok = false;  // one grid, one region
            ++j;
        }
        const LrDev &d = lrd[orb_lr[order[i]]];
        const int I1 = isf_len(d.N[0], d.per[0]), I2 = isf_len(d.N[1], d.per[1]), I3 = isf_len(d.N[2], d.per[2]);
        if (I3 * TX_ * TY_ > 32 * kZThreads) b->density_ok = false;   // accumulators of kd_density
        group_chunk_start.push_back((int)chunk_start.size());
        group_rho.push_back(b->pot_off[order[i]]);
        group_n.push_back(I1 * I2 * I3);
        p.max_group_n = std::max(p.max_group_n, I1 * I2 * I3);
        // a group of many orbitals is split in up to 8 chunks (one partial
        // density each) so that its tiles fill the GPU
        const int n = j - i;
        const int nch = std::min(n, std::max(8, (n + kDenChunk - 1) / kDenChunk));
        const int per_chunk = (n + nch - 1) / nch;
        for (int k = i; k < j; k += per_chunk) {
            const int c = (int)chunk_start.size();
            chunk_start.push_back((int)chunk_orbs.size());
            for (int m = k; m < std::min(j, k + per_chunk); ++m) chunk_orbs.push_back(order[m]);
            chunk_part.push_back(den);
            den += (long long)I1 * I2 * I3;
            const int ntx = (I1 + TX_ - 1) / TX_, nty = (I2 + TY_ - 1) / TY_;
            for (int ty = 0; ty < nty; ++ty)
                for (int tx = 0; tx < ntx; ++tx) wd.push_back(make_int4(c, tx * TX_, ty * TY_, 0));
        }
        i = j;
    }
    chunk_start.push_back((int)chunk_orbs.size());
    group_chunk_start.push_back((int)chunk_part.size());
    p.nchunk = (int)chunk_part.size();
    p.ngroup = (int)group_rho.size();
    p.part_den_elems = den;
    p.n_workd = (int)wd.size();
    if ((rc = upload(p, lrd, &p.d_lr)) || (rc = upload(p, od, &p.d_orb)) || (rc = upload(p, w13, &p.d_work13)) ||
        (rc = upload(p, s13, &p.d_part_slot13)) || (rc = upload(p, w2, &p.d_work2)) ||
        (rc = upload(p, s2, &p.d_part_slot2)) || (rc = upload(p, w2p, &p.d_work2p)) ||
        (rc = upload(p, s2p, &p.d_part_slot2p)) || (rc = upload(p, wd, &p.d_workd)) ||
        (rc = upload(p, chunk_start, &p.d_chunk_orb_start)) || (rc = upload(p, chunk_orbs, &p.d_chunk_orbs)) ||
        (rc = upload(p, chunk_part, &p.d_chunk_part)) || (rc = upload(p, group_chunk_start, &p.d_group_chunk_start)) ||
        (rc = upload(p, group_rho, &p.d_group_rho)) || (rc = upload(p, group_n, &p.d_group_n)) ||
        (rc = upload(p, orb_off, &p.d_orb_off)) || (rc = upload(p, orb_len, &p.d_orb_len))) {
        wvlh_batch_destroy(b);
        return fail(rc);
    }
    *out = b;
    return WVLH_OK;
}

extern "C" int wvlh_batch_destroy(wvlh_batch *b)
{
    if (!b) return WVLH_OK;
    for (void *q : b->plan.owned) cudaFree(q);
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

static size_t sm_limit()
{
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return (size_t)v;
}

extern "C" int wvlh_locham_batched(wvlh_batch *b, int precision, const void *psi, const void *pot, void *hpsi,
                                   double *ekin, double *epot, int accumulate)
{
    if (!b || !psi || !pot || !hpsi || (precision != 32 && precision != 64)) return fail(WVLH_ERR_ARG);
    wvlh_ctx *c = b->ctx;
    CK(cudaSetDevice(c->device));
    const Plan &p = b->plan;
    const int fp = precision == 64;
    const size_t lim = sm_limit() - 1024;
    if (p.smem13[fp] > lim || p.smem2[fp] > lim) return fail(WVLH_ERR_TOO_LARGE);
    int rc;
    if ((rc = c->scratch.ensure(p.scratch_elems * (fp ? 8 : 4))) ||
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
    if (!b || !psi || !hfac || !rho || (precision != 32 && precision != 64)) return fail(WVLH_ERR_ARG);
    if (!b->density_ok) return fail(WVLH_ERR_UNSUPPORTED);
    wvlh_ctx *c = b->ctx;
    CK(cudaSetDevice(c->device));
    const Plan &p = b->plan;
    const int fp = precision == 64;
    const size_t lim = sm_limit() - 1024;
    if (p.smem13[fp] > lim || p.smem2[fp] > lim) return fail(WVLH_ERR_TOO_LARGE);
    int rc;
    if ((rc = c->scratch.ensure(p.scratch_elems * (fp ? 8 : 4))) ||
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
    wvlh_ctx *c = b->ctx;
    CK(cudaSetDevice(c->device));
    const Plan &p = b->plan;
    const int fp = precision == 64;
    const size_t lim = sm_limit() - 1024;
    if (p.smem13[fp] > lim || p.smem2[fp] > lim) return fail(WVLH_ERR_TOO_LARGE);
    const size_t es = fp ? 8 : 4;
    const size_t nv = (size_t)p.psi_total * es;
    int rc;
    if ((rc = c->scratch.ensure(p.scratch_elems * es)) || (rc = c->cg_r.ensure(nv)) || (rc = c->cg_d.ensure(nv)) ||
        (rc = c->cg_ad.ensure(nv)) || (rc = c->cg_scal.ensure(sizeof(double) * (size_t)p.norb * (5 + 16))))
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
size_t overlap_workspace_bytes(int norb, long long K, int nsm);
template <class TI>
cudaError_t launch_overlap(int norb, long long K, long long ld, const TI *psi, double *S, double *work, int nsm,
                           cudaStream_t st);
}  // namespace wvlh

extern "C" int wvlh_overlap(wvlh_ctx *c, int precision, int norb, int64_t K, int64_t ld, const void *psi, double *S)
{
    if (!c || !psi || !S || norb <= 0 || K <= 0 || ld < K || (precision != 32 && precision != 64))
        return fail(WVLH_ERR_ARG);
    CK(cudaSetDevice(c->device));
    int nsm = 0;
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
    int rc;
    if ((rc = c->ov_work.ensure(overlap_workspace_bytes(norb, K, nsm)))) return fail(rc);
    cudaError_t e = precision == 64
                        ? launch_overlap<double>(norb, K, ld, (const double *)psi, S, (double *)c->ov_work.p, nsm,
                                                 c->stream)
                        : launch_overlap<float>(norb, K, ld, (const float *)psi, S, (double *)c->ov_work.p, nsm,
                                                c->stream);
    CK(e);
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

extern "C" int wvlh_locham_batched_host(wvlh_batch *b, int precision, const void *psi, const void *pot, void *hpsi,
                                        double *ekin, double *epot)
{
    if (!b || !psi || !pot || !hpsi || (precision != 32 && precision != 64)) return fail(WVLH_ERR_ARG);
    wvlh_ctx *c = b->ctx;
    CK(cudaSetDevice(c->device));
    const size_t es = precision == 32 ? 4 : 8;
    const size_t npsi = (size_t)b->plan.psi_total * es, npot = (size_t)pot_extent(b) * es;
    const size_t ne = sizeof(double) * b->plan.norb;
    int rc;
    if ((rc = c->io_psi.ensure(npsi)) || (rc = c->io_hpsi.ensure(npsi)) || (rc = c->io_pot.ensure(npot)) ||
        (rc = c->io_e.ensure(2 * ne)))
        return fail(rc);
    CK(cudaMemcpyAsync(c->io_psi.p, psi, npsi, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->io_pot.p, pot, npot, cudaMemcpyHostToDevice, c->stream));
    double *de = (double *)c->io_e.p;
    rc = wvlh_locham_batched(b, precision, c->io_psi.p, c->io_pot.p, c->io_hpsi.p, de, de + b->plan.norb, 0);
    if (rc) return rc;
    CK(cudaMemcpyAsync(hpsi, c->io_hpsi.p, npsi, cudaMemcpyDeviceToHost, c->stream));
    if (ekin) CK(cudaMemcpyAsync(ekin, de, ne, cudaMemcpyDeviceToHost, c->stream));
    if (epot) CK(cudaMemcpyAsync(epot, de + b->plan.norb, ne, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
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
        const int nvc = b->nvc[l], nvf = b->nvf[l];
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
        CK(plain_uncompress(0, dims, b->nsc[l], nvc, b->d_keyg_c[l], b->d_keyv_c[l], b->nsf[l], nvf,
                            b->d_keyg_f[l], b->d_keyv_f[l], W3, W3 + nvc, W0, nullptr, nb, ncomp, ncomp, ni, st));
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
        const double h1 = 0.5 * b->hgrid[3 * l], h2 = 0.5 * b->hgrid[3 * l + 1], h3 = 0.5 * b->hgrid[3 * l + 2];
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
        CK(plain_uncompress(1, dims, b->nsc[l], nvc, b->d_keyg_c[l], b->d_keyv_c[l], b->nsf[l], nvf,
                            b->d_keyg_f[l], b->d_keyv_f[l], W2, W2 + nvc, W1, nullptr, nb, ncomp, ncomp, ni, st));
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
