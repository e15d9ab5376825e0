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
// pairing of segments), built once per atom at creation and flattened into a
// table of (psi value, projector value) offsets.  Three kernels:
//   k_nl_dot:    one CTA per (atom, block of kOrbBlock orbitals), threads over
//                the atom's common values: c = <p|psi>, fixed-order
//                reductions (deterministic);
//   k_nl_coeff:  one CTA per orbital: hc = h c per atom, eproj = sum c.hc;
//                hc is written block-transposed, the kUpdBlock orbitals of a
//                block contiguous per coefficient;
//   k_nl_update: one warp per (grid row, block of kUpdBlock orbitals).  A run
//                lies in one grid row (keys are runs along x) and a row's psi
//                values are contiguous, so rows partition psi: lanes take the
//                row's values, add sum_i hc_i p_i of every atom reaching the
//                value (atoms in order) and write each value once; the block's
//                hc of one coefficient arrive as 16-byte broadcast loads.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
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
constexpr int kProjChunk = 4;  // projectors summed per pass over an atom's runs
// orbital blocks: each projector value loaded serves a block's orbitals;
// smaller blocks (more resident warps) measured slower
constexpr int kOrbBlock = 8;   // orbitals per CTA (dot)
constexpr int kUpdBlock = 16;  // orbitals per warp (update), hc block width

struct NlAtom {
    int nproj;
    int nval;       // common values (fine points count 7)
    int val0;       // first entry of the atom in the value table
    int c0;         // first coefficient of the atom in an orbital's c / hc row
    long long proj; // first projector value in the coefficient block
    int ld_p;       // values of one projector (nvctr_c + 7 nvctr_f)
    int h0;         // first coefficient of the atom's h matrix
};

// one run of common points: psi value offset, projector value offset (fine
// runs already at nvctr_c + 7 point), number of values
struct NlRun {
    int w, p, n, atom;
};

__global__ void __launch_bounds__(256) k_nl_dot(const NlAtom *__restrict__ atoms, const int2 *__restrict__ vals,
                                                const double *__restrict__ proj, const double *__restrict__ psi,
                                                long long ld, int norb, int ctot, double *__restrict__ cf)
{
    __shared__ double red[kOrbBlock * kProjChunk][8];
    const NlAtom at = atoms[blockIdx.x];
    const int o0 = blockIdx.y * kOrbBlock;
    const int nob = min(kOrbBlock, norb - o0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const double *pa = proj + at.proj;
    const int2 *v0 = vals + at.val0;
    for (int p0 = 0; p0 < at.nproj; p0 += kProjChunk) {
        const int np = min(kProjChunk, at.nproj - p0);
        double s[kOrbBlock][kProjChunk];
#pragma unroll
        for (int b = 0; b < kOrbBlock; ++b)
#pragma unroll
            for (int k = 0; k < kProjChunk; ++k) s[b][k] = 0.0;
        // the next value's offsets are loaded one iteration ahead
        int2 qn = threadIdx.x < at.nval ? v0[threadIdx.x] : make_int2(0, 0);
        for (int i = threadIdx.x; i < at.nval; i += blockDim.x) {
            const int2 q = qn;   // (psi value, projector value)
            if (i + (int)blockDim.x < at.nval) qn = v0[i + blockDim.x];
            double pv[kProjChunk];
#pragma unroll
            for (int k = 0; k < kProjChunk; ++k) pv[k] = k < np ? pa[(size_t)(p0 + k) * at.ld_p + q.y] : 0.0;
#pragma unroll
            for (int b = 0; b < kOrbBlock; ++b) {
                if (b < nob) {
                    const double v = psi[(size_t)(o0 + b) * ld + q.x];
#pragma unroll
                    for (int k = 0; k < kProjChunk; ++k) s[b][k] = fma(v, pv[k], s[b][k]);
                }
            }
        }
#pragma unroll
        for (int b = 0; b < kOrbBlock; ++b)
#pragma unroll
            for (int k = 0; k < kProjChunk; ++k) {
                double v = s[b][k];
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
                if (lane == 0) red[b * kProjChunk + k][warp] = v;
            }
        __syncthreads();
        if (threadIdx.x < kOrbBlock * kProjChunk) {
            const int b = threadIdx.x / kProjChunk, k = threadIdx.x % kProjChunk;
            if (b < nob && k < np) {
                double v = 0.0;
                for (int w = 0; w < nw; ++w) v += red[threadIdx.x][w];
                cf[(size_t)(o0 + b) * ctot + at.c0 + p0 + k] = v;
            }
        }
        __syncthreads();
    }
}

// hc = h c per atom; eproj = sum over atoms of c . hc (thread t takes atoms
// t, t + 128, ...; the thread sums are added in thread order: deterministic).
// hc[(o / kUpdBlock) ctot + c][o % kUpdBlock]: a block's orbitals contiguous
__global__ void __launch_bounds__(128) k_nl_coeff(int natoms, const NlAtom *__restrict__ atoms,
                                                  const double *__restrict__ hmat, int ctot,
                                                  const double *__restrict__ cf, double *__restrict__ hc,
                                                  double *__restrict__ eproj)
{
    __shared__ double ea[128];
    const int o = blockIdx.x;
    const double *c = cf + (size_t)o * ctot;
    double *h = hc + (size_t)(o / kUpdBlock) * ctot * kUpdBlock + o % kUpdBlock;
    double e = 0.0;   // thread t: atoms t, t + 128, ...
    for (int a = threadIdx.x; a < natoms; a += blockDim.x) {
        const NlAtom at = atoms[a];
        double ep = 0.0;
        for (int i = 0; i < at.nproj; ++i) {
            const double *hr = hmat + at.h0 + (size_t)i * at.nproj;
            double v = 0.0;
            for (int j = 0; j < at.nproj; ++j) v = fma(hr[j], c[at.c0 + j], v);
            h[(size_t)(at.c0 + i) * kUpdBlock] = v;
            ep = fma(c[at.c0 + i], v, ep);
        }
        e += ep;
    }
    ea[threadIdx.x] = e;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < (int)blockDim.x; ++k) t += ea[k];
        eproj[o] = t;
    }
}

// a run as the update reads it: projector base such that proj + pb + wv is
// the value of the run's first projector at psi value wv; psi range [w, w+n);
// the atom's projector count, projector stride and first coefficient
struct NlRunMeta {
    long long pb;
    int w, n, np, ldp, cc, pad;
};

// runs c .. min(c + 32, e1) - 1 of a row into the warp's metadata slots
__device__ __forceinline__ void nl_stage_runs(const NlRun *__restrict__ rrun, const NlAtom *__restrict__ atoms,
                                              int c, int e1, int lane, NlRunMeta *mw)
{
    __syncwarp();
    if (lane < e1 - c) {
        const NlRun r = rrun[c + lane];
        const NlAtom at = atoms[r.atom];
        NlRunMeta m;
        m.pb = at.proj + r.p - r.w;
        m.w = r.w;
        m.n = r.n;
        m.np = at.nproj;
        m.ldp = at.ld_p;
        m.cc = at.c0;
        m.pad = 0;
        mw[lane] = m;
    }
    __syncwarp();
}

// one warp per (row group, orbital block): rows[g] .. rows[g+1] index the
// row-sorted run list (atoms in order within a row); rowv[g] = the row's first
// psi value and value count.  The row's runs (32 at a time) are staged in
// shared memory once per warp, so the value loop reads no run or atom record
// from memory; each lane prefetches its value's hpsi before the sums.  hc is
// block-transposed (k_nl_coeff), zero for the orbitals past norb in the last
// block, so every FMA is unconditional
__global__ void __launch_bounds__(256, 2) k_nl_update(int ngroups, const int *__restrict__ rows,
                                                      const int2 *__restrict__ rowv, const NlRun *__restrict__ rrun,
                                                      const NlAtom *__restrict__ atoms,
                                                      const double *__restrict__ proj, int norb, int ctot,
                                                      const double *__restrict__ hc, long long ld,
                                                      double *__restrict__ hpsi)
{
    __shared__ NlRunMeta meta[8][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = blockIdx.x * (blockDim.x >> 5) + warp;
    if (g >= ngroups) return;   // whole warps leave together
    const int o0 = blockIdx.y * kUpdBlock;
    const int nob = min(kUpdBlock, norb - o0);
    const int2 rv = rowv[g];
    const int e0 = rows[g], e1 = rows[g + 1];
    const double2 *hblk = reinterpret_cast<const double2 *>(hc + (size_t)blockIdx.y * ctot * kUpdBlock);
    NlRunMeta *mw = meta[warp];
    const bool one = e1 - e0 <= 32;
    if (one) nl_stage_runs(rrun, atoms, e0, e1, lane, mw);
    for (int ub = 0; ub < rv.y; ub += 32) {   // warp-uniform: every lane stages
        const int u = ub + lane;
        const bool act = u < rv.y;
        const int wv = rv.x + u;
        double old[kUpdBlock], v[kUpdBlock];
#pragma unroll
        for (int b = 0; b < kUpdBlock; ++b) {
            old[b] = (act && b < nob) ? hpsi[(size_t)(o0 + b) * ld + wv] : 0.0;
            v[b] = 0.0;
        }
        for (int c = e0; c < e1; c += 32) {
            if (!one) nl_stage_runs(rrun, atoms, c, e1, lane, mw);
            const int cnt = min(32, e1 - c);
            if (!act) continue;
            for (int k = 0; k < cnt; ++k) {
                const int t = wv - mw[k].w;
                if (t < 0 || t >= mw[k].n) continue;
                const NlRunMeta m = mw[k];
                const double *pa = proj + m.pb + wv;
                const double2 *hb = hblk + (size_t)m.cc * (kUpdBlock / 2);
                for (int i = 0; i < m.np; ++i) {
                    const double p = pa[(size_t)i * m.ldp];
#pragma unroll
                    for (int q = 0; q < kUpdBlock / 2; ++q) {
                        const double2 h = hb[(size_t)i * (kUpdBlock / 2) + q];
                        v[2 * q] = fma(h.x, p, v[2 * q]);
                        v[2 * q + 1] = fma(h.y, p, v[2 * q + 1]);
                    }
                }
            }
        }
        if (act) {
#pragma unroll
            for (int b = 0; b < kUpdBlock; ++b)
                if (b < nob) hpsi[(size_t)(o0 + b) * ld + wv] = old[b] + v[b];
        }
    }
}

}  // namespace wvlh

using namespace wvlh;

struct wvlh_nlpsp {
    wvlh_ctx *ctx = nullptr;
    const wvlh_region *psi_region = nullptr;
    int natoms = 0, ctot = 0, ngroups = 0;
    void *mem = nullptr;   // atoms, value table, runs by row, row index and ranges, projectors, h
    NlAtom *d_atoms = nullptr;
    int2 *d_vals = nullptr, *d_rowv = nullptr;
    NlRun *d_rrun = nullptr;
    int *d_rows = nullptr;
    double *d_proj = nullptr, *d_h = nullptr;
    DevBuf cf, hc;         // c (a row of ctot per orbital) and hc (block-transposed)
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
    nl->cf.release();
    nl->hc.release();
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
    const wvlh_region *w = psi_region;
    std::vector<NlAtom> at(natoms);
    long long nproj_vals = 0, nh = 0;
    int nseg_tot = 0, ctot = 0;
    for (int a = 0; a < natoms; ++a) {
        const wvlh_region *pr = proj_regions[a];
        if (!pr || pr->device != ctx->device || nproj[a] < 0 || nproj[a] > kMaxProj) return nl_fail(WVLH_ERR_ARG);
        for (int k = 0; k < 3; ++k)
            if (pr->lr.N[k] != w->lr.N[k]) return nl_fail(WVLH_ERR_ARG);  // one box
        NlAtom &t = at[a];
        t.nproj = nproj[a];
        t.c0 = ctot;
        t.proj = nproj_vals;
        t.ld_p = pr->lr.nvctr_c + 7 * pr->lr.nvctr_f;
        t.h0 = (int)nh;
        ctot += t.nproj;
        nseg_tot += pr->lr.nseg_c + pr->lr.nseg_f;
        nproj_vals += (long long)t.nproj * t.ld_p;
        nh += (long long)t.nproj * t.nproj;
    }
    if (cudaSetDevice(ctx->device) != cudaSuccess) return nl_fail(WVLH_ERR_CUDA);
    cudaStream_t st = ctx->stream;
    // the runs of every projector segment (k_wpdot_runs: psi is a, the
    // projector b) and the projectors' segment starts, brought to the host
    std::vector<int4> hr(nseg_tot > 0 ? nseg_tot : 1);
    std::vector<uint32_t> kg(2 * (size_t)(nseg_tot > 0 ? nseg_tot : 1));
    if (nseg_tot > 0) {
        int4 *d_tmp = nullptr;
        if (cudaMalloc(&d_tmp, sizeof(int4) * nseg_tot) != cudaSuccess) return nl_fail(WVLH_ERR_NOMEM);
        cudaError_t e = cudaSuccess;
        int s0 = 0;
        for (int a = 0; a < natoms && e == cudaSuccess; ++a) {
            const wvlh_region *pr = proj_regions[a];
            const int nc = pr->lr.nseg_c, nf = pr->lr.nseg_f;
            if (nc > 0)
                k_wpdot_runs<<<(nc + 255) / 256, 256, 0, st>>>(w->lr.nseg_c, w->keyg_c, w->keyv_c, nc, pr->keyg_c,
                                                                pr->keyv_c, d_tmp + s0);
            if (nf > 0)
                k_wpdot_runs<<<(nf + 255) / 256, 256, 0, st>>>(w->lr.nseg_f, w->keyg_f, w->keyv_f, nf, pr->keyg_f,
                                                                pr->keyv_f, d_tmp + s0 + nc);
            e = cudaGetLastError();
            if (e == cudaSuccess && nc > 0)
                e = cudaMemcpyAsync(kg.data() + 2 * (size_t)s0, pr->keyg_c, 8 * (size_t)nc, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess && nf > 0)
                e = cudaMemcpyAsync(kg.data() + 2 * (size_t)(s0 + nc), pr->keyg_f, 8 * (size_t)nf,
                                    cudaMemcpyDeviceToHost, st);
            s0 += nc + nf;
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(hr.data(), d_tmp, sizeof(int4) * nseg_tot, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        cudaFree(d_tmp);
        if (e != cudaSuccess) return nl_fail(WVLH_ERR_CUDA);
    }
    // runs in values (fine points carry 7); per atom the flat table of its
    // common values (psi offset, projector offset); the same runs by grid row
    // (coarse rows, then fine rows), atoms in order within a row
    const int N1 = w->lr.N[0], nrow = w->lr.N[1] * w->lr.N[2];
    std::vector<NlRun> runs;
    std::vector<int2> vals;
    std::vector<std::pair<long long, int>> order;   // (row key, index in runs)
    int s0 = 0;
    for (int a = 0; a < natoms; ++a) {
        const wvlh_region *pr = proj_regions[a];
        const int nc = pr->lr.nseg_c, nf = pr->lr.nseg_f;
        at[a].val0 = (int)vals.size();
        for (int q = 0; q < nc + nf; ++q) {
            const int4 r = hr[s0 + q];
            if (r.z <= 0) continue;
            const bool fine = q >= nc;
            NlRun x;
            x.w = fine ? w->lr.nvctr_c + 7 * r.x : r.x;
            x.p = fine ? pr->lr.nvctr_c + 7 * r.y : r.y;
            x.n = fine ? 7 * r.z : r.z;
            x.atom = a;
            for (int t = 0; t < x.n; ++t) vals.push_back(make_int2(x.w + t, x.p + t));
            const long long row = (long long)(kg[2 * (size_t)(s0 + q)] - 1) / N1 + (fine ? nrow : 0);
            order.emplace_back(row, (int)runs.size());
            runs.push_back(x);
        }
        at[a].nval = (int)vals.size() - at[a].val0;
        s0 += nc + nf;
    }
    if (vals.size() > (size_t)0x7fffffff) return nl_fail(WVLH_ERR_TOO_LARGE);
    std::stable_sort(order.begin(), order.end(),
                     [](const std::pair<long long, int> &u, const std::pair<long long, int> &v) { return u.first < v.first; });
    std::vector<NlRun> rrun;
    std::vector<int> rows;
    std::vector<int2> rowv;   // first psi value of the row's runs, values spanned
    for (size_t k = 0; k < order.size(); ++k) {
        const NlRun &x = runs[order[k].second];
        if (k == 0 || order[k].first != order[k - 1].first) {
            rows.push_back((int)k);
            rowv.push_back(make_int2(x.w, x.n));
        } else {
            int2 &rv = rowv.back();
            const int lo = std::min(rv.x, x.w), hi = std::max(rv.x + rv.y, x.w + x.n);
            rv = make_int2(lo, hi - lo);
        }
        rrun.push_back(x);
    }
    rows.push_back((int)order.size());
    const int ngroups = (int)rows.size() - 1;
    auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t n_r = runs.empty() ? 1 : runs.size(), n_v = vals.empty() ? 1 : vals.size();
    const size_t o_atoms = 0, o_vals = up(sizeof(NlAtom) * (natoms > 0 ? natoms : 1));
    const size_t o_rrun = o_vals + up(sizeof(int2) * n_v);
    const size_t o_rows = o_rrun + up(sizeof(NlRun) * n_r);
    const size_t o_rowv = o_rows + up(sizeof(int) * rows.size());
    const size_t o_proj = o_rowv + up(sizeof(int2) * (rowv.empty() ? 1 : rowv.size()));
    const size_t o_h = o_proj + up(sizeof(double) * (nproj_vals > 0 ? nproj_vals : 1));
    const size_t total = o_h + up(sizeof(double) * (nh > 0 ? nh : 1));
    wvlh_nlpsp *nl = new wvlh_nlpsp();
    nl->ctx = ctx;
    nl->psi_region = psi_region;
    nl->natoms = natoms;
    nl->ctot = ctot;
    nl->ngroups = ngroups;
    if (cudaMalloc(&nl->mem, total) != cudaSuccess) {
        delete nl;
        return nl_fail(WVLH_ERR_NOMEM);
    }
    unsigned char *base = (unsigned char *)nl->mem;
    nl->d_atoms = (NlAtom *)(base + o_atoms);
    nl->d_vals = (int2 *)(base + o_vals);
    nl->d_rrun = (NlRun *)(base + o_rrun);
    nl->d_rows = (int *)(base + o_rows);
    nl->d_rowv = (int2 *)(base + o_rowv);
    nl->d_proj = (double *)(base + o_proj);
    nl->d_h = (double *)(base + o_h);
    cudaError_t e = cudaSuccess;
    if (natoms > 0) e = cudaMemcpyAsync(nl->d_atoms, at.data(), sizeof(NlAtom) * natoms, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && !vals.empty())
        e = cudaMemcpyAsync(nl->d_vals, vals.data(), sizeof(int2) * vals.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && !rowv.empty())
        e = cudaMemcpyAsync(nl->d_rowv, rowv.data(), sizeof(int2) * rowv.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && !rrun.empty())
        e = cudaMemcpyAsync(nl->d_rrun, rrun.data(), sizeof(NlRun) * rrun.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(nl->d_rows, rows.data(), sizeof(int) * rows.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && nproj_vals > 0)
        e = cudaMemcpyAsync(nl->d_proj, proj, sizeof(double) * nproj_vals, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess && nh > 0) e = cudaMemcpyAsync(nl->d_h, hij, sizeof(double) * nh, cudaMemcpyHostToDevice, st);
    // the host tables are copied before returning
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
    if (!nl || norb < 0 || norb > 65535 * kOrbBlock || (norb > 0 && (!psi || !hpsi || !eproj)))
        return nl_fail(WVLH_ERR_ARG);
    if (ld < wvlh_region_psi_size(nl->psi_region)) return nl_fail(WVLH_ERR_ARG);
    if (norb == 0) return WVLH_OK;
    if (cudaSetDevice(nl->ctx->device) != cudaSuccess) return nl_fail(WVLH_ERR_CUDA);
    cudaStream_t st = nl->ctx->stream;
    const int nblk = (norb + kOrbBlock - 1) / kOrbBlock;
    if (nl->natoms == 0 || nl->ctot == 0) {
        if (cudaMemsetAsync(eproj, 0, sizeof(double) * norb, st) != cudaSuccess) return nl_fail(WVLH_ERR_CUDA);
        return WVLH_OK;
    }
    const size_t cb = sizeof(double) * (size_t)norb * nl->ctot;
    const int nub = (norb + kUpdBlock - 1) / kUpdBlock;
    const size_t hb = sizeof(double) * (size_t)nub * kUpdBlock * nl->ctot;
    int rc;
    if ((rc = nl->cf.ensure(cb)) || (rc = nl->hc.ensure(hb))) return nl_fail(rc);
    double *cf = (double *)nl->cf.p, *hc = (double *)nl->hc.p;
    // the last block's columns past norb stay zero
    if (norb % kUpdBlock && cudaMemsetAsync(hc + (size_t)(nub - 1) * kUpdBlock * nl->ctot, 0,
                                            sizeof(double) * kUpdBlock * nl->ctot, st) != cudaSuccess)
        return nl_fail(WVLH_ERR_CUDA);
    k_nl_dot<<<dim3(nl->natoms, nblk), 256, 0, st>>>(nl->d_atoms, nl->d_vals, nl->d_proj, psi, ld, norb, nl->ctot, cf);
    k_nl_coeff<<<norb, 128, 0, st>>>(nl->natoms, nl->d_atoms, nl->d_h, nl->ctot, cf, hc, eproj);
    if (nl->ngroups > 0)
        k_nl_update<<<dim3((nl->ngroups + 7) / 8, nub), 256, 0, st>>>(nl->ngroups, nl->d_rows, nl->d_rowv, nl->d_rrun,
                                                                     nl->d_atoms, nl->d_proj, norb, nl->ctot, hc, ld,
                                                                     hpsi);
    if (cudaGetLastError() != cudaSuccess) return nl_fail(WVLH_ERR_CUDA);
    return WVLH_OK;
}
