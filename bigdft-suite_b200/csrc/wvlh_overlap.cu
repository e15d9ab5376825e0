// Overlap matrix S = Psi^T Psi of the orbitals on FP64 tensor cores.
//
// The reference forms the lower triangle with syrk('L','T', norb, nvctrp)
// over its component-distributed coefficients (getOverlap,
// wfn_opt/orthogonality.f90:2624-2697, syrk at :2675) and sums it over ranks.
// Here psi is the batch layout (orbital rows of length K, row stride ld) and
// S is computed as lower-triangular 64x64 tiles, split over K so that every
// SM has work; each split writes an FP64 partial tile and a second kernel sums
// the splits in a fixed order (deterministic) and mirrors the tile into the
// upper triangle.
//
// The same kernel forms the subspace matrix L = Psi (H Psi)^T of two panels
// (TWO: every tile of the square, B rows from the second panel, no mirror):
// the Lagrange multipliers of orthoconstraint (orthogonality.f90:375-625,
// subspace_matrix :196-224, gemm('T','N')).
//
// Main loop: a 2-stage cp.async ring stages 64 x 32 slices of the two orbital
// panels in their storage type (16-byte copies when rows are 16-byte aligned),
// so the loads of slice s+1 overlap the MMAs of slice s; at 74 KB (FP64) three
// CTAs fit an SM.  The contraction uses
// mma.sync m16n8k16 with FP64 operands (the largest FP64 tensor-core shape of
// sm_90+/sm_100a; the tcgen05 family has no FP64 kind): 4 warps, each a 32 x 32
// sub-tile = 2 x 4 MMA tiles; FP32 rows are widened when fragments are read.
#include <cuda_runtime.h>

#include <cstdint>

namespace wvlh {

constexpr int OV_BM = 64;       // tile edge (rows = orbitals i, cols = orbitals j)
constexpr int OV_BK = 32;       // K slice per pipeline stage
constexpr int OV_STAGES = 2;
constexpr int OV_THREADS = 128;

template <class TI> struct OvLd;   // padded smem row (elements): 16-byte multiple, 2-way bank spread
template <> struct OvLd<double> { static constexpr int v = 36; };
template <> struct OvLd<float> { static constexpr int v = 36; };

__host__ __device__ constexpr size_t overlap_smem_bytes(size_t elem)
{
    return (size_t)2 * OV_STAGES * OV_BM * 36 * elem;
}

// D = A(16x16) B(16x8) + D, FP64.  Fragments (lane = 4 g + t):
// a[i] = A[g + 8 (i & 1)][t + 4 (i >> 1)], b[i] = B[t + 4 i][g],
// c = {D[g][2t], D[g][2t+1], D[g+8][2t], D[g+8][2t+1]}
__device__ __forceinline__ void dmma_16x8x16(double (&c)[4], const double (&a)[8], const double (&b)[4])
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
        "{%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]),
          "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

__device__ __forceinline__ void ov_cp_async(void *dst, const void *src, int bytes, int src_bytes)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    if (bytes == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
    else if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void ov_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void ov_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// tile t of the lower triangle -> (ti, tj), ti >= tj
__device__ __forceinline__ void tri_tile(int t, int &ti, int &tj)
{
    int i = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
    while ((i + 1) * (i + 2) / 2 <= t) ++i;
    while (i * (i + 1) / 2 > t) --i;
    ti = i;
    tj = t - i * (i + 1) / 2;
}

// Stage rows r0.. of a 64 x 32 slice starting at column k0 (zero past ke or norb).
// VEC: bytes per copy (16 when psi rows are 16-byte aligned, else the element size).
template <class TI, int VEC>
__device__ __forceinline__ void ov_stage(TI *dst, const TI *__restrict__ psi, long long ld, int row0, int norb,
                                         long long k0, long long ke)
{
    constexpr int LD = OvLd<TI>::v;
    constexpr int EPV = VEC / (int)sizeof(TI);        // elements per copy
    constexpr int CPR = OV_BK / EPV;                  // copies per row
    for (int e = threadIdx.x; e < OV_BM * CPR; e += OV_THREADS) {
        const int r = e / CPR, c = (e - r * CPR) * EPV;
        const long long k = k0 + c;
        const int row = row0 + r;
        long long nvalid = ke - k;
        nvalid = nvalid < 0 ? 0 : (nvalid > EPV ? EPV : nvalid);
        if (row >= norb) nvalid = 0;
        const TI *src = nvalid ? psi + (size_t)row * ld + k : psi;
        ov_cp_async(dst + r * LD + c, src, VEC, (int)(nvalid * sizeof(TI)));
    }
}

template <class TI, int VEC, bool TWO>
__global__ void __launch_bounds__(OV_THREADS) k_overlap_partial(int norb, long long K, long long ld,
                                                                const TI *__restrict__ psi,
                                                                const TI *__restrict__ psib, int nsplit,
                                                                long long kchunk, double *__restrict__ part)
{
    extern __shared__ __align__(16) unsigned char ov_smem[];
    constexpr int LD = OvLd<TI>::v;
    TI *As = reinterpret_cast<TI *>(ov_smem);
    TI *Bs = As + OV_STAGES * OV_BM * LD;
    const int tile = blockIdx.x / nsplit, split = blockIdx.x % nsplit;
    int ti, tj;
    if (TWO) {
        const int nt = (norb + OV_BM - 1) / OV_BM;
        ti = tile / nt;
        tj = tile - ti * nt;
    } else {
        tri_tile(tile, ti, tj);
    }
    const TI *pb = TWO ? psib : psi;
    const int i0 = ti * OV_BM, j0 = tj * OV_BM;
    const bool diag = !TWO && ti == tj;
    const long long kb = split * kchunk;
    const long long ke = kb + kchunk < K ? kb + kchunk : K;
    const int nk = ke > kb ? (int)((ke - kb + OV_BK - 1) / OV_BK) : 0;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32;   // warp sub-tile origin
    // on a diagonal tile the strictly upper 32 x 32 block is not needed
    const bool idle = diag && wc > wr;
    double acc[2][4][4];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[a][b][q] = 0.0;

#pragma unroll
    for (int s = 0; s < OV_STAGES - 1; ++s) {
        if (s < nk) {
            ov_stage<TI, VEC>(As + s * OV_BM * LD, psi, ld, i0, norb, kb + (long long)s * OV_BK, ke);
            if (!diag) ov_stage<TI, VEC>(Bs + s * OV_BM * LD, pb, ld, j0, norb, kb + (long long)s * OV_BK, ke);
        }
        ov_commit();
    }
    for (int it = 0; it < nk; ++it) {
        ov_wait<OV_STAGES - 2>();
        __syncthreads();   // slice it is visible; slot (it-1) % STAGES is free
        {
            const int s = it + OV_STAGES - 1;
            if (s < nk) {
                const int slot = s % OV_STAGES;
                ov_stage<TI, VEC>(As + slot * OV_BM * LD, psi, ld, i0, norb, kb + (long long)s * OV_BK, ke);
                if (!diag)
                    ov_stage<TI, VEC>(Bs + slot * OV_BM * LD, pb, ld, j0, norb, kb + (long long)s * OV_BK, ke);
            }
            ov_commit();
        }
        const int slot = it % OV_STAGES;
        const TI *Ar = As + slot * OV_BM * LD;
        const TI *Br = (diag ? As : Bs) + slot * OV_BM * LD;
        if (!idle) {
#pragma unroll
            for (int kk = 0; kk < OV_BK; kk += 16) {
                double fa[2][8], fb[4][4];
#pragma unroll
                for (int a = 0; a < 2; ++a)
#pragma unroll
                    for (int i = 0; i < 8; ++i)
                        fa[a][i] = (double)Ar[(wr + 16 * a + g + 8 * (i & 1)) * LD + kk + t + 4 * (i >> 1)];
#pragma unroll
                for (int b = 0; b < 4; ++b)
#pragma unroll
                    for (int i = 0; i < 4; ++i) fb[b][i] = (double)Br[(wc + 8 * b + g) * LD + kk + t + 4 * i];
#pragma unroll
                for (int a = 0; a < 2; ++a)
#pragma unroll
                    for (int b = 0; b < 4; ++b) dmma_16x8x16(acc[a][b], fa[a], fb[b]);
            }
        }
    }
    ov_wait<0>();
    // partial tile, row-major 64x64 (the idle block of a diagonal tile is never read)
    double *out = part + ((size_t)tile * nsplit + split) * OV_BM * OV_BM;
    if (!idle) {
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int r = wr + 16 * a + g;
                const int c = wc + 8 * b + 2 * t;
                out[r * OV_BM + c] = acc[a][b][0];
                out[r * OV_BM + c + 1] = acc[a][b][1];
                out[(r + 8) * OV_BM + c] = acc[a][b][2];
                out[(r + 8) * OV_BM + c + 1] = acc[a][b][3];
            }
    }
}

// one thread per tile element (grid.x tiles, grid.y element blocks): the
// splits are summed in order, so the result does not depend on the grid
template <bool TWO>
__global__ void k_overlap_reduce(int norb, int nsplit, const double *__restrict__ part, double *__restrict__ S)
{
    const int tile = blockIdx.x;
    int ti, tj;
    if (TWO) {
        const int nt = (norb + OV_BM - 1) / OV_BM;
        ti = tile / nt;
        tj = tile - ti * nt;
    } else {
        tri_tile(tile, ti, tj);
    }
    const int e = blockIdx.y * blockDim.x + threadIdx.x;
    if (e >= OV_BM * OV_BM) return;
    const int r = e / OV_BM, c = e - r * OV_BM;
    const int i = ti * OV_BM + r, j = tj * OV_BM + c;
    if (i >= norb || j >= norb || (!TWO && j > i)) return;
    double s = 0.0;
    for (int k = 0; k < nsplit; ++k) s += part[((size_t)tile * nsplit + k) * OV_BM * OV_BM + e];
    S[(size_t)i * norb + j] = s;
    if (!TWO) S[(size_t)j * norb + i] = s;
}

// splits over K: about three CTAs per SM (the 2-stage FP64 ring takes 74 KB)
static int overlap_tiles(int norb, bool two)
{
    const int nt = (norb + OV_BM - 1) / OV_BM;
    return two ? nt * nt : nt * (nt + 1) / 2;
}

int overlap_split(int norb, long long K, int nsm, bool two)
{
    const int ntile = overlap_tiles(norb, two);
    // three CTAs fit an SM (72 KB of shared memory each in FP64): as many
    // splits as fill those slots without starting a second, nearly empty wave
    // (rounding up put 450 CTAs on 444 slots at 256 orbitals: the last six ran
    // alone and the tensor pipes idled a third of the time)
    int nsplit = 3 * nsm / ntile;
    const long long maxs = (K + OV_BK - 1) / OV_BK;
    if (nsplit > maxs) nsplit = (int)maxs;
    return nsplit < 1 ? 1 : nsplit;
}

size_t overlap_workspace_bytes(int norb, long long K, int nsm, bool two)
{
    return sizeof(double) * (size_t)overlap_tiles(norb, two) * overlap_split(norb, K, nsm, two) * OV_BM * OV_BM;
}

// S = psi psi^T (psib null: lower tiles, mirrored) or psi psib^T (every tile)
template <class TI>
cudaError_t launch_overlap(int norb, long long K, long long ld, const TI *psi, const TI *psib, double *S,
                           double *work, int nsm, cudaStream_t st)
{
    const bool two = psib != nullptr;
    const int ntile = overlap_tiles(norb, two);
    const int nsplit = overlap_split(norb, K, nsm, two);
    long long kchunk = (K + nsplit - 1) / nsplit;
    kchunk = (kchunk + OV_BK - 1) / OV_BK * OV_BK;
    const size_t smem = overlap_smem_bytes(sizeof(TI));
    // 16-byte copies need every row start (and the bases) on a 16-byte boundary
    const bool vec16 = ((uintptr_t)psi % 16 == 0) && (!two || (uintptr_t)psib % 16 == 0) &&
                       ((ld * (long long)sizeof(TI)) % 16 == 0);
    cudaError_t e;
    auto go = [&](auto k) -> cudaError_t {
        cudaError_t r;
        if ((r = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem))) return r;
        k<<<ntile * nsplit, OV_THREADS, smem, st>>>(norb, K, ld, psi, psib, nsplit, kchunk, work);
        return cudaGetLastError();
    };
    if (two) e = vec16 ? go(k_overlap_partial<TI, 16, true>) : go(k_overlap_partial<TI, (int)sizeof(TI), true>);
    else e = vec16 ? go(k_overlap_partial<TI, 16, false>) : go(k_overlap_partial<TI, (int)sizeof(TI), false>);
    if (e) return e;
    if (two) k_overlap_reduce<true><<<dim3(ntile, OV_BM * OV_BM / 256), 256, 0, st>>>(norb, nsplit, work, S);
    else k_overlap_reduce<false><<<dim3(ntile, OV_BM * OV_BM / 256), 256, 0, st>>>(norb, nsplit, work, S);
    return cudaGetLastError();
}
template cudaError_t launch_overlap<double>(int, long long, long long, const double *, const double *, double *,
                                            double *, int, cudaStream_t);

// ---------------------------------------------------------------------------
// Panel apply C = beta C + alpha M Psi (norb x K, FP64) with a small
// norb x norb matrix M, the psi-sized step of the orthonormalisation and of
// the Lagrange-multiplier update:
//   Cholesky   Psi <- L^-1 Psi     (dpotrf, dtrtri, dtrmm; orthogonality.f90:2351-2366)
//   Loewdin    Psi <- S^-1/2 Psi   (dsyev, then the product; :2486)
//   subspace   HPsi <- HPsi - L^T Psi (subspace_update, :254-271)
// Each CTA forms a 64 (i) x 64 (k) tile of C, contracting over j in slices
// of 32 staged by a 2-stage cp.async ring (16-byte copies): M[i0.., j0..]
// as 64 x 32 and Psi[j0.., k0..] as 32 x 64, on the same FP64 tensor-core
// MMA as the overlap (4 warps, 32 x 32 each).  LOWER: M is lower triangular,
// so the slices past the tile's last row are skipped (the TRMM of dtrmm).
// The contraction over j runs in a fixed order: results do not depend on the
// grid.  C must not alias Psi.
constexpr int PA_LDB = 64 + 4;   // Psi slice row: 64 k + 4 (conflict-free fragment loads)

// VEC: 16-byte copies (two doubles) when norb, ld and the bases allow,
// else one double per copy
template <int VEC>
__device__ __forceinline__ void pa_stage(double *As, double *Bs, const double *__restrict__ M, int norb,
                                         const double *__restrict__ psi, long long ld, long long K, int i0, int j0,
                                         long long k0)
{
    constexpr int LD = OvLd<double>::v;
    constexpr int E = VEC / 8;   // doubles per copy
    // M slice: 64 rows x 32 columns
    for (int e = threadIdx.x; e < OV_BM * (OV_BK / E); e += OV_THREADS) {
        const int r = e / (OV_BK / E), c = (e - r * (OV_BK / E)) * E;
        const int i = i0 + r, j = j0 + c;
        const int nvalid = (i < norb) ? (norb - j >= E ? E : (norb - j > 0 ? norb - j : 0)) : 0;
        const double *src = nvalid ? M + (size_t)i * norb + j : M;
        ov_cp_async(As + r * LD + c, src, VEC, nvalid * 8);
    }
    // Psi slice: 32 rows x 64 columns
    for (int e = threadIdx.x; e < OV_BK * (OV_BM / E); e += OV_THREADS) {
        const int r = e / (OV_BM / E), c = (e - r * (OV_BM / E)) * E;
        const int j = j0 + r;
        const long long k = k0 + c;
        long long nv = K - k;
        nv = nv < 0 ? 0 : (nv > E ? E : nv);
        if (j >= norb) nv = 0;
        const double *src = nv ? psi + (size_t)j * ld + k : psi;
        ov_cp_async(Bs + r * PA_LDB + c, src, VEC, (int)(nv * 8));
    }
}

template <bool LOWER, int VEC>
__global__ void __launch_bounds__(OV_THREADS) k_panel_apply(int norb, long long K, long long ld,
                                                            const double *__restrict__ M,
                                                            const double *__restrict__ psi, double alpha,
                                                            double beta, double *__restrict__ C)
{
    extern __shared__ __align__(16) unsigned char pa_smem[];
    constexpr int LD = OvLd<double>::v;
    constexpr int ASZ = OV_BM * LD, BSZ = OV_BK * PA_LDB;
    double *As = reinterpret_cast<double *>(pa_smem);
    double *Bs = As + OV_STAGES * ASZ;
    const long long k0 = (long long)blockIdx.x * OV_BM;
    const int i0 = blockIdx.y * OV_BM;
    // contraction range: all of j, or j <= the tile's last row (lower M)
    const int jend = LOWER ? min(norb, i0 + OV_BM) : norb;
    const int nj = (jend + OV_BK - 1) / OV_BK;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32;
    double acc[2][4][4];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[a][b][q] = 0.0;
    if (nj > 0) pa_stage<VEC>(As, Bs, M, norb, psi, ld, K, i0, 0, k0);
    ov_commit();
    for (int it = 0; it < nj; ++it) {
        ov_wait<0>();
        __syncthreads();   // slice it is visible; the other slot is free
        if (it + 1 < nj) {
            const int slot = (it + 1) % OV_STAGES;
            pa_stage<VEC>(As + slot * ASZ, Bs + slot * BSZ, M, norb, psi, ld, K, i0, (it + 1) * OV_BK, k0);
        }
        ov_commit();
        const int slot = it % OV_STAGES;
        const double *Ar = As + slot * ASZ;
        const double *Br = Bs + slot * BSZ;
#pragma unroll
        for (int kk = 0; kk < OV_BK; kk += 16) {
            double fa[2][8], fb[4][4];
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int i = 0; i < 8; ++i) fa[a][i] = Ar[(wr + 16 * a + g + 8 * (i & 1)) * LD + kk + t + 4 * (i >> 1)];
#pragma unroll
            for (int b = 0; b < 4; ++b)
#pragma unroll
                for (int i = 0; i < 4; ++i) fb[b][i] = Br[(kk + t + 4 * i) * PA_LDB + wc + 8 * b + g];
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) dmma_16x8x16(acc[a][b], fa[a], fb[b]);
        }
    }
    ov_wait<0>();
    // C rows i, columns k: two neighbouring columns per fragment row
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int i = i0 + wr + 16 * a + g + 8 * h;
                const long long k = k0 + wc + 8 * b + 2 * t;
                if (i >= norb) continue;
                double *c = C + (size_t)i * ld + k;
                const double v0 = alpha * acc[a][b][2 * h], v1 = alpha * acc[a][b][2 * h + 1];
                if (VEC == 16 && k + 1 < K) {
                    double2 o = make_double2(v0, v1);
                    if (beta != 0.0) {
                        const double2 old = *reinterpret_cast<const double2 *>(c);
                        o.x = fma(beta, old.x, v0);
                        o.y = fma(beta, old.y, v1);
                    }
                    *reinterpret_cast<double2 *>(c) = o;
                } else {
                    if (k < K) c[0] = beta != 0.0 ? fma(beta, c[0], v0) : v0;
                    if (k + 1 < K) c[1] = beta != 0.0 ? fma(beta, c[1], v1) : v1;
                }
            }
}

size_t panel_apply_smem_bytes() { return sizeof(double) * OV_STAGES * (OV_BM * OvLd<double>::v + OV_BK * PA_LDB); }

// C = beta C + alpha M psi; psi, C rows of K at row stride ld
cudaError_t launch_panel_apply(int norb, long long K, long long ld, const double *M, int lower, double alpha,
                               const double *psi, double beta, double *C, cudaStream_t st)
{
    const size_t smem = panel_apply_smem_bytes();
    const dim3 grid((unsigned)((K + OV_BM - 1) / OV_BM), (unsigned)((norb + OV_BM - 1) / OV_BM));
    auto go = [&](auto k) -> cudaError_t {
        cudaError_t r;
        if ((r = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem))) return r;
        k<<<grid, OV_THREADS, smem, st>>>(norb, K, ld, M, psi, alpha, beta, C);
        return cudaGetLastError();
    };
    // two doubles per copy and store when every row start is on 16 bytes
    const bool v16 = !(norb % 2) && !(ld % 2) && !((uintptr_t)M % 16) && !((uintptr_t)psi % 16) &&
                     !((uintptr_t)C % 16);
    if (v16) return lower ? go(k_panel_apply<true, 16>) : go(k_panel_apply<false, 16>);
    return lower ? go(k_panel_apply<true, 8>) : go(k_panel_apply<false, 8>);
}
template cudaError_t launch_overlap<float>(int, long long, long long, const float *, const float *, double *,
                                           double *, int, cudaStream_t);

}  // namespace wvlh
