// Compressed scalar products between vectors on different keys of one box
// (the reference's wpdot, wavelib/scalprod.f90:3222-3420).
//
// Step 1 (k_wpdot_runs): one thread per segment of b finds, by binary search
// over a's segment starts, the a segment it is paired with and the run of
// common points, exactly as the reference's loop does: the first a segment
// meeting [max(b start, first a start), b end]; b segments that follow the
// first one starting past a's last segment start get no run (the reference's
// search index has then run past the end).  A run is {a offset, b offset,
// length} in points (fine points carry 7 components).
// Step 2 (k_wpdot_dot): one CTA per (a vector, b vector) pair sums the runs
// in FP64, warps over runs, lanes over points, fixed-order block reduction
// (deterministic).
#include <cuda_runtime.h>
#include <stdint.h>

#include "wvlh_common.cuh"

namespace wvlh {

__global__ void k_wpdot_runs(int nseg_a, const uint32_t *__restrict__ kg_a, const uint32_t *__restrict__ kv_a,
                             int nseg_b, const uint32_t *__restrict__ kg_b, const uint32_t *__restrict__ kv_b,
                             int4 *__restrict__ runs)
{
    const int ib = blockIdx.x * blockDim.x + threadIdx.x;
    if (ib >= nseg_b) return;
    int4 r = make_int4(0, 0, 0, 0);
    if (nseg_a > 0) {
        const long long kbs = kg_b[2 * ib], kbe = kg_b[2 * ib + 1];
        const long long first = kg_a[0], last = kg_a[2 * (nseg_a - 1)];
        const bool skipped = ib > 0 && (long long)kg_b[2 * (ib - 1)] > last;
        if (!skipped) {
            long long jb0 = kbs > first ? kbs : first;
            int lo = 0, hi = nseg_a - 1;   // last a segment with start <= jb0
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if ((long long)kg_a[2 * mid] <= jb0) lo = mid; else hi = mid - 1;
            }
            int s = lo;
            bool ok = true;
            if ((long long)kg_a[2 * s + 1] < jb0) {   // a segment ends before: try the next one
                s += 1;
                ok = s < nseg_a && (long long)kg_a[2 * s] <= kbe;
                if (ok) jb0 = kg_a[2 * s];
            }
            if (ok) {
                const long long ea = kg_a[2 * s + 1];
                const long long n = (kbe < ea ? kbe : ea) - jb0 + 1;
                if (n > 0) {
                    r.x = (int)(kv_a[s] - 1 + (jb0 - (long long)kg_a[2 * s]));
                    r.y = (int)(kv_b[ib] - 1 + (jb0 - kbs));
                    r.z = (int)n;
                }
            }
        }
    }
    runs[ib] = r;
}

template <class T>
__global__ void __launch_bounds__(256) k_wpdot_dot(int nrun_c, int nrun_f, const int4 *__restrict__ runs,
                                                   const T *__restrict__ a, long long lda, int nvc_a,
                                                   const T *__restrict__ b, long long ldb, int nvc_b, int nb,
                                                   double *__restrict__ out)
{
    __shared__ double red[32];
    const int j = blockIdx.x, i = blockIdx.y;
    const T *ai = a + (size_t)i * lda, *bj = b + (size_t)j * ldb;
    const T *af = ai + nvc_a, *bf = bj + nvc_b;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double s = 0.0;
    for (int q = warp; q < nrun_c + nrun_f; q += nw) {
        const int4 r = runs[q];
        if (q < nrun_c) {
            for (int t = lane; t < r.z; t += 32) s += (double)ai[r.x + t] * (double)bj[r.y + t];
        } else {
            const T *pa = af + 7 * (size_t)r.x, *pb = bf + 7 * (size_t)r.y;
            for (int t = lane; t < 7 * r.z; t += 32) s += (double)pa[t] * (double)pb[t];
        }
    }
    const double tot = block_sum(s, red);
    if (threadIdx.x == 0) out[(size_t)i * nb + j] = tot;
}

// runs: nseg_bc + nseg_bf int4 (device scratch)
template <class T>
cudaError_t launch_wpdot(int nseg_ac, const uint32_t *kg_ac, const uint32_t *kv_ac, int nseg_af,
                         const uint32_t *kg_af, const uint32_t *kv_af, int nvc_a, int nseg_bc, const uint32_t *kg_bc,
                         const uint32_t *kv_bc, int nseg_bf, const uint32_t *kg_bf, const uint32_t *kv_bf, int nvc_b,
                         int na, const T *a, long long lda, int nb, const T *b, long long ldb, double *out,
                         int4 *runs, cudaStream_t st)
{
    if (nseg_bc > 0)
        k_wpdot_runs<<<(nseg_bc + 255) / 256, 256, 0, st>>>(nseg_ac, kg_ac, kv_ac, nseg_bc, kg_bc, kv_bc, runs);
    if (nseg_bf > 0)
        k_wpdot_runs<<<(nseg_bf + 255) / 256, 256, 0, st>>>(nseg_af, kg_af, kv_af, nseg_bf, kg_bf, kv_bf,
                                                             runs + nseg_bc);
    k_wpdot_dot<T><<<dim3(nb, na), 256, 0, st>>>(nseg_bc, nseg_bf, runs, a, lda, nvc_a, b, ldb, nvc_b, nb, out);
    return cudaGetLastError();
}

template cudaError_t launch_wpdot<float>(int, const uint32_t *, const uint32_t *, int, const uint32_t *,
                                         const uint32_t *, int, int, const uint32_t *, const uint32_t *, int,
                                         const uint32_t *, const uint32_t *, int, int, const float *, long long, int,
                                         const float *, long long, double *, int4 *, cudaStream_t);
template cudaError_t launch_wpdot<double>(int, const uint32_t *, const uint32_t *, int, const uint32_t *,
                                          const uint32_t *, int, int, const uint32_t *, const uint32_t *, int,
                                          const uint32_t *, const uint32_t *, int, int, const double *, long long,
                                          int, const double *, long long, double *, int4 *, cudaStream_t);

}  // namespace wvlh
