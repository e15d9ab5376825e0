// Overlap matrix S = Psi^T Psi of the orbitals on FP64 tensor cores.
//
// The reference forms the lower triangle with syrk('L','T', norb, nvctrp)
// over its component-distributed coefficients (getOverlap,
// wfn_opt/orthogonality.f90:2624-2697, syrk at :2675) and sums it over ranks.
// Here psi is the batch layout (orbital rows of length K, row stride ld) and
// S is computed as lower-triangular 64x64 tiles, split over K so that every
// SM has work; each split writes an FP64 partial tile and a second kernel sums
// the splits in a fixed order (deterministic) and mirrors the tile into the
// upper triangle.  The contraction uses mma.sync m8n8k4 with FP64 operands
// (the FP64 tensor-core instruction of sm_100a; the tcgen05 family has no
// FP64 kind).  FP32 inputs are widened to FP64 when staged in shared memory.
#include <cuda_runtime.h>

#include <cstdint>

namespace wvlh {

constexpr int OV_BM = 64;      // tile edge (rows = orbitals i, cols = orbitals j)
constexpr int OV_BK = 32;      // K slice staged per iteration
constexpr int OV_LD = OV_BK + 2;
constexpr int OV_THREADS = 128;

__device__ __forceinline__ void dmma_8x8x4(double (&c)[2], double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

// tile t of the lower triangle -> (ti, tj), ti >= tj
__device__ __forceinline__ void tri_tile(int t, int &ti, int &tj)
{
    int i = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
    while ((i + 1) * (i + 2) / 2 <= t) ++i;
    while (i * (i + 1) / 2 > t) --i;
    ti = i;
    tj = t - i * (i + 1) / 2;
}

template <class TI>
__global__ void __launch_bounds__(OV_THREADS) k_overlap_partial(int norb, long long K, long long ld,
                                                                const TI *__restrict__ psi, int nsplit,
                                                                long long kchunk, double *__restrict__ part)
{
    __shared__ double As[OV_BM * OV_LD];
    __shared__ double Bs[OV_BM * OV_LD];
    const int tile = blockIdx.x / nsplit, split = blockIdx.x % nsplit;
    int ti, tj;
    tri_tile(tile, ti, tj);
    const int i0 = ti * OV_BM, j0 = tj * OV_BM;
    const bool diag = ti == tj;
    const long long kb = split * kchunk;
    const long long ke = kb + kchunk < K ? kb + kchunk : K;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32;   // warp sub-tile origin
    double acc[4][4][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;

    for (long long k0 = kb; k0 < ke; k0 += OV_BK) {
        // stage A (rows i0..i0+63) and B (rows j0..), zero outside
        for (int e = threadIdx.x; e < OV_BM * OV_BK; e += OV_THREADS) {
            const int r = e / OV_BK, c = e - r * OV_BK;
            const long long k = k0 + c;
            const int ia = i0 + r, jb = j0 + r;
            As[r * OV_LD + c] = (ia < norb && k < ke) ? (double)psi[ia * ld + k] : 0.0;
            if (!diag) Bs[r * OV_LD + c] = (jb < norb && k < ke) ? (double)psi[jb * ld + k] : 0.0;
        }
        __syncthreads();
        const double *Bsrc = diag ? As : Bs;
#pragma unroll
        for (int kk = 0; kk < OV_BK; kk += 4) {
            double fa[4], fb[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) fa[a] = As[(wr + 8 * a + (lane >> 2)) * OV_LD + kk + (lane & 3)];
#pragma unroll
            for (int b = 0; b < 4; ++b) fb[b] = Bsrc[(wc + 8 * b + (lane >> 2)) * OV_LD + kk + (lane & 3)];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) dmma_8x8x4(acc[a][b], fa[a], fb[b]);
        }
        __syncthreads();
    }
    // partial tile, row-major 64x64
    double *out = part + ((size_t)tile * nsplit + split) * OV_BM * OV_BM;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int r = wr + 8 * a + (lane >> 2);
            const int c = wc + 8 * b + 2 * (lane & 3);
            out[r * OV_BM + c] = acc[a][b][0];
            out[r * OV_BM + c + 1] = acc[a][b][1];
        }
}

__global__ void k_overlap_reduce(int norb, int nsplit, const double *__restrict__ part, double *__restrict__ S)
{
    const int tile = blockIdx.x;
    int ti, tj;
    tri_tile(tile, ti, tj);
    for (int e = threadIdx.x; e < OV_BM * OV_BM; e += blockDim.x) {
        const int r = e / OV_BM, c = e - r * OV_BM;
        const int i = ti * OV_BM + r, j = tj * OV_BM + c;
        if (i >= norb || j >= norb || j > i) continue;
        double s = 0.0;
        for (int k = 0; k < nsplit; ++k) s += part[((size_t)tile * nsplit + k) * OV_BM * OV_BM + e];
        S[(size_t)i * norb + j] = s;
        S[(size_t)j * norb + i] = s;
    }
}

int overlap_split(int norb, long long K, int nsm)
{
    const int nt = (norb + OV_BM - 1) / OV_BM;
    const int ntile = nt * (nt + 1) / 2;
    int nsplit = (4 * nsm + ntile - 1) / ntile;
    const long long maxs = (K + OV_BK - 1) / OV_BK;
    if (nsplit > maxs) nsplit = (int)maxs;
    return nsplit < 1 ? 1 : nsplit;
}

size_t overlap_workspace_bytes(int norb, long long K, int nsm)
{
    const int nt = (norb + OV_BM - 1) / OV_BM;
    return sizeof(double) * (size_t)(nt * (nt + 1) / 2) * overlap_split(norb, K, nsm) * OV_BM * OV_BM;
}

template <class TI>
cudaError_t launch_overlap(int norb, long long K, long long ld, const TI *psi, double *S, double *work, int nsm,
                           cudaStream_t st)
{
    const int nt = (norb + OV_BM - 1) / OV_BM;
    const int ntile = nt * (nt + 1) / 2;
    const int nsplit = overlap_split(norb, K, nsm);
    long long kchunk = (K + nsplit - 1) / nsplit;
    kchunk = (kchunk + OV_BK - 1) / OV_BK * OV_BK;
    k_overlap_partial<TI><<<ntile * nsplit, OV_THREADS, 0, st>>>(norb, K, ld, psi, nsplit, kchunk, work);
    k_overlap_reduce<<<ntile, 256, 0, st>>>(norb, nsplit, work, S);
    return cudaGetLastError();
}
template cudaError_t launch_overlap<double>(int, long long, long long, const double *, double *, double *, int,
                                            cudaStream_t);
template cudaError_t launch_overlap<float>(int, long long, long long, const float *, double *, double *, int,
                                           cudaStream_t);

}  // namespace wvlh
