// Nonlocal pseudopotential projectors: hpsi += sum_atoms sum_ij p_i h_ij <p_j|psi>
// and the projector energy per orbital (NonLocalHamiltonianApplication,
// hpsiortho.f90:1044-1125; DFT_PSP_projectors_iter_apply,
// modules/psp_projectors.f90:585-712).
//
// The reference packs psi onto each projector's points through a mask of
// common segments (count_wblas_segs / fill_wblas_segs,
// locregs/scalar_product.f90:1012-1187), takes the scalar products with a
// GEMM, applies the atom's coefficient matrix, and adds the projector
// combination back through the same mask (waxpy_mask_unpack, :953).  Here the
// masks are the runs of the compressed scalar product (k_wpdot_runs, the same
// pairing of segments), built once per atom at creation; one CTA per orbital
// walks the atoms in order:
//   c_i = sum over run points of psi * p_i   (warps over runs, lanes over
//         points, fixed-order block reduction: deterministic),
//   hc  = h c, eproj += c . hc,
//   psi-side points += sum_i hc_i p_i          (each point by one thread).
// One CTA owns an orbital, so atoms whose projectors overlap never race.
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../../include/wvlh.h"
#include "wvlh_common.cuh"
#include "wvlh_internal.h"
#include "wvlh_objects.h"

namespace wvlh {
__global__ void k_wpdot_runs(int nseg_a, const uint32_t *__restrict__ kg_a, const uint32_t *__restrict__ kv_a,
                             int nseg_b, const uint32_t *__restrict__ kg_b, const uint32_t *__restrict__ kv_b,
                             int4 *__restrict__ runs);
void set_last_error(int code);

constexpr int kMaxProj = 32;   // projectors per atom
constexpr int kProjChunk = 8;  // projectors summed per pass over an atom's runs

struct NlAtom {
    int nproj;
    int nrun_c, nrun_f;  // coarse runs, then fine runs
    int run0;            // first run in the run table
    long long proj;      // first projector value in the coefficient block
    int nvc_p;           // coarse values of one projector (its fine part follows)
    int ld_p;            // values of one projector (nvctr_c + 7 nvctr_f)
    int h0;              // first coefficient of the atom's h matrix
    int pad;
};

// one CTA per orbital, atoms in order
__global__ void __launch_bounds__(256) k_nlpsp_apply(int natoms, const NlAtom *__restrict__ atoms,
                                                     const int4 *__restrict__ runs,
                                                     const double *__restrict__ proj,
                                                     const double *__restrict__ hmat, const double *__restrict__ psi,
                                                     long long ld, int nvc_w, double *__restrict__ hpsi,
                                                     double *__restrict__ eproj)
{
    __shared__ double red[kProjChunk][8];   // per-warp partial sums of one chunk
    __shared__ double c[kMaxProj], hc[kMaxProj];
    const int o = blockIdx.x;
    const double *w = psi + (size_t)o * ld;
    double *hw = hpsi + (size_t)o * ld;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double e = 0.0;
    for (int a = 0; a < natoms; ++a) {
        const NlAtom at = atoms[a];
        const int4 *r = runs + at.run0;
        const double *pa = proj + at.proj;
        const int nr = at.nrun_c + at.nrun_f;
        // c_i = <p_i | psi>, kProjChunk projectors per pass over the runs
        for (int p0 = 0; p0 < at.nproj; p0 += kProjChunk) {
            double s[kProjChunk];
#pragma unroll
            for (int k = 0; k < kProjChunk; ++k) s[k] = 0.0;
            const int np = min(kProjChunk, at.nproj - p0);
            for (int q = warp; q < nr; q += nw) {
                const int4 run = r[q];
                const bool fine = q >= at.nrun_c;
                const int n = fine ? 7 * run.z : run.z;
                const double *wp = fine ? w + nvc_w + 7 * (size_t)run.x : w + run.x;
                const size_t pb = fine ? (size_t)at.nvc_p + 7 * (size_t)run.y : (size_t)run.y;
                for (int t = lane; t < n; t += 32) {
                    const double v = wp[t];
#pragma unroll
                    for (int k = 0; k < kProjChunk; ++k)
                        if (k < np) s[k] = fma(v, pa[(size_t)(p0 + k) * at.ld_p + pb + t], s[k]);
                }
            }
#pragma unroll
            for (int k = 0; k < kProjChunk; ++k) {
                double v = s[k];
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
                if (lane == 0) red[k][warp] = v;
            }
            __syncthreads();
            if (threadIdx.x < np) {
                double v = 0.0;
                for (int k = 0; k < nw; ++k) v += red[threadIdx.x][k];
                c[p0 + threadIdx.x] = v;
            }
            __syncthreads();
        }
        // hc = h c and the atom's energy c . hc
        if (threadIdx.x < at.nproj) {
            const double *h = hmat + at.h0 + (size_t)threadIdx.x * at.nproj;
            double v = 0.0;
            for (int j = 0; j < at.nproj; ++j) v = fma(h[j], c[j], v);
            hc[threadIdx.x] = v;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double ea = 0.0;
            for (int i = 0; i < at.nproj; ++i) ea = fma(c[i], hc[i], ea);
            e += ea;
        }
        // psi-side points += sum_i hc_i p_i: the runs of one atom are disjoint
        // on the psi side, so every point has one writer
        for (int q = warp; q < nr; q += nw) {
            const int4 run = r[q];
            const bool fine = q >= at.nrun_c;
            const int n = fine ? 7 * run.z : run.z;
            double *hp = fine ? hw + nvc_w + 7 * (size_t)run.x : hw + run.x;
            const size_t pb = fine ? (size_t)at.nvc_p + 7 * (size_t)run.y : (size_t)run.y;
            for (int t = lane; t < n; t += 32) {
                double v = 0.0;
                for (int i = 0; i < at.nproj; ++i) v = fma(hc[i], pa[(size_t)i * at.ld_p + pb + t], v);
                hp[t] += v;
            }
        }
        __syncthreads();   // the next atom may touch the same points and reuses c, hc
    }
    if (threadIdx.x == 0) eproj[o] = e;
}

}  // namespace wvlh

using namespace wvlh;

struct wvlh_nlpsp {
    wvlh_ctx *ctx = nullptr;
    const wvlh_region *psi_region = nullptr;
    int natoms = 0;
    void *mem = nullptr;   // atoms, runs, projectors, h matrices
    NlAtom *d_atoms = nullptr;
    int4 *d_runs = nullptr;
    double *d_proj = nullptr, *d_h = nullptr;
};

static int nl_fail(int code)
{
    set_last_error(code);
    return code;
}

extern "C" int wvlh_nlpsp_destroy(wvlh_nlpsp *nl)
{
    if (!nl) return WVLH_OK;
    cudaSetDevice(nl->ctx->device);
    cudaStreamSynchronize(nl->ctx->stream);
    if (nl->mem) cudaFree(nl->mem);
    delete nl;
    return WVLH_OK;
}

extern "C" int wvlh_nlpsp_create(wvlh_ctx *ctx, const wvlh_region *psi_region, int natoms,
                                 const wvlh_region *const *proj_regions, const int *nproj, const double *proj,
                                 const double *hij, wvlh_nlpsp **out)
{
    if (!ctx || !psi_region || natoms < 0 || (natoms > 0 && (!proj_regions || !nproj || !proj || !hij)) || !out)
        return nl_fail(WVLH_ERR_ARG);
    *out = nullptr;
    if (psi_region->device != ctx->device) return nl_fail(WVLH_ERR_ARG);
    std::vector<NlAtom> at(natoms);
    long long nproj_vals = 0, nh = 0;
    int nruns = 0;
    for (int a = 0; a < natoms; ++a) {
        const wvlh_region *pr = proj_regions[a];
        if (!pr || pr->device != ctx->device || nproj[a] < 0 || nproj[a] > kMaxProj) return nl_fail(WVLH_ERR_ARG);
        for (int k = 0; k < 3; ++k)
            if (pr->lr.N[k] != psi_region->lr.N[k]) return nl_fail(WVLH_ERR_ARG);  // one box
        NlAtom &t = at[a];
        t.nproj = nproj[a];
        t.nrun_c = pr->lr.nseg_c;
        t.nrun_f = pr->lr.nseg_f;
        t.run0 = nruns;
        t.proj = nproj_vals;
        t.nvc_p = pr->lr.nvctr_c;
        t.ld_p = pr->lr.nvctr_c + 7 * pr->lr.nvctr_f;
        t.h0 = (int)nh;
        t.pad = 0;
        nruns += t.nrun_c + t.nrun_f;
        nproj_vals += (long long)t.nproj * t.ld_p;
        nh += (long long)t.nproj * t.nproj;
    }
    auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t o_atoms = 0, o_runs = up(sizeof(NlAtom) * (natoms > 0 ? natoms : 1));
    const size_t o_proj = o_runs + up(sizeof(int4) * (nruns > 0 ? nruns : 1));
    const size_t o_h = o_proj + up(sizeof(double) * (nproj_vals > 0 ? nproj_vals : 1));
    const size_t total = o_h + up(sizeof(double) * (nh > 0 ? nh : 1));
    if (cudaSetDevice(ctx->device) != cudaSuccess) return nl_fail(WVLH_ERR_CUDA);
    wvlh_nlpsp *nl = new wvlh_nlpsp();
    nl->ctx = ctx;
    nl->psi_region = psi_region;
    nl->natoms = natoms;
    if (cudaMalloc(&nl->mem, total) != cudaSuccess) {
        delete nl;
        return nl_fail(WVLH_ERR_NOMEM);
    }
    unsigned char *base = (unsigned char *)nl->mem;
    nl->d_atoms = (NlAtom *)(base + o_atoms);
    nl->d_runs = (int4 *)(base + o_runs);
    nl->d_proj = (double *)(base + o_proj);
    nl->d_h = (double *)(base + o_h);
    cudaStream_t st = ctx->stream;
    cudaError_t e = cudaSuccess;
    if (natoms > 0) e = cudaMemcpyAsync(nl->d_atoms, at.data(), sizeof(NlAtom) * natoms, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && nproj_vals > 0)
        e = cudaMemcpyAsync(nl->d_proj, proj, sizeof(double) * nproj_vals, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess && nh > 0) e = cudaMemcpyAsync(nl->d_h, hij, sizeof(double) * nh, cudaMemcpyHostToDevice, st);
    // runs: psi (a) against each projector (b), coarse then fine
    const wvlh_region *w = psi_region;
    for (int a = 0; a < natoms && e == cudaSuccess; ++a) {
        const wvlh_region *pr = proj_regions[a];
        int4 *r = nl->d_runs + at[a].run0;
        if (pr->lr.nseg_c > 0)
            k_wpdot_runs<<<(pr->lr.nseg_c + 255) / 256, 256, 0, st>>>(w->lr.nseg_c, w->keyg_c, w->keyv_c,
                                                                      pr->lr.nseg_c, pr->keyg_c, pr->keyv_c, r);
        if (pr->lr.nseg_f > 0)
            k_wpdot_runs<<<(pr->lr.nseg_f + 255) / 256, 256, 0, st>>>(w->lr.nseg_f, w->keyg_f, w->keyv_f,
                                                                      pr->lr.nseg_f, pr->keyg_f, pr->keyv_f,
                                                                      r + pr->lr.nseg_c);
        e = cudaGetLastError();
    }
    // hij is a host array: finish its copy before returning
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        wvlh_nlpsp_destroy(nl);
        return nl_fail(WVLH_ERR_CUDA);
    }
    *out = nl;
    return WVLH_OK;
}

extern "C" int wvlh_nlpsp_apply(wvlh_nlpsp *nl, int norb, const double *psi, int64_t ld, double *hpsi, double *eproj)
{
    if (!nl || norb < 0 || (norb > 0 && (!psi || !hpsi || !eproj))) return nl_fail(WVLH_ERR_ARG);
    if (ld < wvlh_region_psi_size(nl->psi_region)) return nl_fail(WVLH_ERR_ARG);
    if (norb == 0) return WVLH_OK;
    if (cudaSetDevice(nl->ctx->device) != cudaSuccess) return nl_fail(WVLH_ERR_CUDA);
    k_nlpsp_apply<<<norb, 256, 0, nl->ctx->stream>>>(nl->natoms, nl->d_atoms, nl->d_runs, nl->d_proj, nl->d_h, psi,
                                                     ld, nl->psi_region->lr.nvctr_c, hpsi, eproj);
    if (cudaGetLastError() != cudaSuccess) return nl_fail(WVLH_ERR_CUDA);
    return WVLH_OK;
}
