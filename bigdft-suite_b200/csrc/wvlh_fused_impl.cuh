// Fused, batched local Hamiltonian (Hpsi, E_kin, E_pot), density and
// preconditioner operator for many orbitals and many localisation regions,
// FP32 or FP64.
//
// The reference applies locham to one orbital at a time as 13 full-array
// passes (uncompress, 3x syn, 3x MF, xV, 3x MF^T, 3x kinetic, 3x ana,
// compress: orbitals/daubisf.f90:214-331, locregs/locreg_operations.f90:2502-2937,
// OpenCL/Hamiltonian.c:105-172).  Because every 1D operator acts on one
// axis, the chain factorises as
//     Hpsi = A_x A_y [ Mt_x Mt_y Z1 + Z2 + (K_x + K_y) P ]
//     P  = S_x S_y psi,    Q = M_x M_y P                       (plane kernel K1)
//     Z1 = A_z Mt_z V M_z S_z Q,   Z2 = A_z K_z S_z P            (z kernel K2)
// (S syn, A ana, M magic filter, K kinetic) so that each kernel keeps a whole
// xy-plane or a whole z-pencil tile in shared memory and chains its 1D passes
// there.  E_pot = sum V r^2 comes from K2; E_kin = sum_d <X|K_d X> with
// X = S^3 psi: the z part from K2 on X itself, the x,y parts from K3 on P
// (<X|K_x X> = <P|K_x P> because S_z is an isometry).  Energies are reduced
// in FP64 into per-CTA partial slots and summed in a fixed order.
//
// The same kernels in MODE_LOCDEN give the density rho += hfac (M^3 S^3 psi)^2
// (OpenCL/Density.c:37-55, sumrho.f90:472-577) through K1 (Q only) and a
// z-kernel that loops over the orbitals sharing a density grid, and in
// MODE_PRECOND the preconditioner operator D^-1/2 A (c + T) S D^-1/2 of
// OpenCL/Preconditioner.c:98-128 through K1 (scaled gather, P only), the
// kinetic chain of K2 and K3 (Z2 + c P + (K_x+K_y) P, scaled scatter).
//
// This file is the implementation shared by the translation units
// wvlh_fused_f32.cu and wvlh_fused_f64.cu, which instantiate the launchers of
// one precision each (the two compile in parallel); the common out-of-line
// helpers are compiled in the FP64 unit (WVLH_FUSED_COMMON).
#pragma once
#include <cuda_runtime.h>

#include <cstring>
#include <type_traits>

#include "wvlh_common.cuh"
#include "wvlh_internal.h"
#include "wvlh_pairs.cuh"
#include "wvlh_tma.cuh"

namespace wvlh {

constexpr int TX = TX_;
constexpr int TY = TY_;
constexpr int TC = TX * TY;
// alignment of the z kernel's tile buffer (a TMA box destination), and the
// bytes its launches add to the two tile buffers: the block-sum slots and
// the TMA barrier
constexpr int kZAlign = 128;
constexpr int kZExtra = 32 * 8 + 16;

template <class T> struct Seg;
template <> struct Seg<float> { static constexpr int v = 8; };
template <> struct Seg<double> { static constexpr int v = 4; };

struct Dims {
    int N1, N2, N3, p1, p2, p3;
    int H1, H2;  // offsets of the wavelet halves of the coarse x and y lines
    int G1, G2, G3, F1, F2, F3, I1, I2, I3;
    // allper: the batch is known to be periodic in every direction, which lets
    // the compiler drop the free-boundary variants from the kernel
    __device__ __forceinline__ Dims(const LrDev &L, bool allper)
    {
        N1 = L.N[0]; N2 = L.N[1]; N3 = L.N[2];
        p1 = allper ? 1 : L.per[0];
        p2 = allper ? 1 : L.per[1];
        p3 = allper ? 1 : L.per[2];
        H1 = half_off(N1); H2 = half_off(N2);
        G1 = coarse_width(N1); G2 = coarse_width(N2); G3 = 2 * N3;
        F1 = fine_len(N1, p1); F2 = fine_len(N2, p2); F3 = fine_len(N3, p3);
        I1 = isf_len(N1, p1); I2 = isf_len(N2, p2); I3 = isf_len(N3, p3);
    }
    // plane buffer A: rows() lines (y) of pitch() points (x).  The second
    // buffer B holds P (F2 rows of pitch()) or a transposed plane: the lines
    // along x of a pass, each of the y length `len` of its plane, at pitch
    // pitchT(len) — sized per pass, so B is no larger than its largest use.
    __device__ __forceinline__ int pitch() const { return vec_pitch(max(G1, max(F1, I1))); }
    __device__ __forceinline__ int rows() const { return max(G2, max(F2, I2)); }
    __device__ __forceinline__ static int pitchT(int len) { return vec_pitch(len); }
};

__device__ __forceinline__ LineGeom rows_geom(int nrows, int pitch)
{
    return LineGeom{nrows, pitch, 1, pitch, 1};
}
__device__ __forceinline__ LineGeom cols_geom(int ncols, int pitch)
{
    return LineGeom{ncols, 1, pitch, 1, pitch};
}
// lines read with unit stride, output written transposed: point q of line l
// goes to dst[q * dst_pitch + l], so the next pass again reads unit stride
__device__ __forceinline__ LineGeom xpose_geom(int nlines, int src_pitch, int dst_pitch)
{
    return LineGeom{nlines, src_pitch, 1, 1, dst_pitch};
}

// fine component c=1..7 of psi_f -> (s1,s2,s3) bits (wavelib/un-compress.f90:930-936)
__device__ __forceinline__ int fs1(int c) { return c & 1; }
__device__ __forceinline__ int fs2(int c) { return (c >> 1) & 1; }
__device__ __forceinline__ int fs3(int c) { return (c >> 2) & 1; }

// Preconditioner diagonal D^-1/2 per component k = s1 + 2 s2 + 4 s3: GPUscal0..7
// of OpenCL/Uncompress.c:380-470 with h = hgrid/2 (the host passes 0.5*hgrid).
__device__ __forceinline__ double prec_scal(const LrDev &L, double c, int k)
{
    double s = c;
    for (int d = 0; d < 3; ++d) {
        const double h = 0.5 * L.hgrid[d];
        s += (((k >> d) & 1) ? WVL_B2 : WVL_A2) * (0.125 / (h * h));
    }
    return 1.0 / sqrt(s);
}

// Scatter the compressed coefficients of wavelet-basis plane kz into the
// (G2 x G1, pitch) buffer A, which must be zero.  Wavelet components sit at
// x + half_off(N1) and y + half_off(N2).  psi points at [psi_c|psi_f]; sc (8
// factors) scales each component when non-null.
template <class T, class TI, int S3>
__device__ __forceinline__ void gather_plane_s(T *A, int pitch, const LrDev &L, int i3, const TI *psi, const T *sc)
{
    const int H1 = half_off(L.N[0]), H2 = half_off(L.N[1]);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (!S3) {
        const T s0 = sc ? sc[0] : T(1);
        const int a = L.plane_c[i3], b = L.plane_c[i3 + 1];
        for (int sg = a + warp; sg < b; sg += nw) {
            const int4 d = L.seg_c[sg];
            for (int t = lane; t < d.z; t += 32) A[d.y * pitch + d.x + t] = (T)psi[d.w + t] * s0;
        }
    }
    const TI *pf = psi + L.nvctr_c;
    const int a = L.plane_f[i3], b = L.plane_f[i3 + 1];
    for (int sg = a + warp; sg < b; sg += nw) {
        const int4 d = L.seg_f[sg];
        for (int t = lane; t < d.z; t += 32) {
            const TI *src = pf + 7 * (size_t)(d.w + t);
#pragma unroll
            for (int c = 1; c <= 7; ++c) {
                if (fs3(c) != S3) continue;
                A[(fs2(c) * H2 + d.y) * pitch + fs1(c) * H1 + d.x + t] = (T)src[c - 1] * (sc ? sc[c] : T(1));
            }
        }
    }
}

// the z component s3 of a plane is uniform over the CTA: one copy of the
// component loop per s3, so no instruction is issued for the other half
template <class T, class TI>
__device__ void gather_plane(T *A, int pitch, const LrDev &L, int kz, const TI *psi, const T *sc)
{
    if (kz >= L.N[2]) gather_plane_s<T, TI, 1>(A, pitch, L, kz - L.N[2], psi, sc);
    else gather_plane_s<T, TI, 0>(A, pitch, L, kz, psi, sc);
}

// Inverse of gather_plane: write (or add into) the compressed output.
template <class T, class TO, int S3>
__device__ __forceinline__ void scatter_plane_s(const T *A, int pitch, const LrDev &L, int i3, TO *out, bool accumulate,
                                                const T *sc)
{
    const int H1 = half_off(L.N[0]), H2 = half_off(L.N[1]);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (!S3) {
        const T s0 = sc ? sc[0] : T(1);
        const int a = L.plane_c[i3], b = L.plane_c[i3 + 1];
        for (int sg = a + warp; sg < b; sg += nw) {
            const int4 d = L.seg_c[sg];
            for (int t = lane; t < d.z; t += 32) {
                const TO v = (TO)(A[d.y * pitch + d.x + t] * s0);
                out[d.w + t] = accumulate ? out[d.w + t] + v : v;
            }
        }
    }
    TO *pf = out + L.nvctr_c;
    const int a = L.plane_f[i3], b = L.plane_f[i3 + 1];
    for (int sg = a + warp; sg < b; sg += nw) {
        const int4 d = L.seg_f[sg];
        for (int t = lane; t < d.z; t += 32) {
            const size_t i = 7 * (size_t)(d.w + t);
            TO *dst = pf + i;
#pragma unroll
            for (int c = 1; c <= 7; ++c) {
                if (fs3(c) != S3) continue;
                const TO v = (TO)(A[(fs2(c) * H2 + d.y) * pitch + fs1(c) * H1 + d.x + t] * (sc ? sc[c] : T(1)));
                dst[c - 1] = accumulate ? dst[c - 1] + v : v;
            }
        }
    }
}

template <class T, class TO>
__device__ void scatter_plane(const T *A, int pitch, const LrDev &L, int kz, TO *out, bool accumulate, const T *sc)
{
    if (kz >= L.N[2]) scatter_plane_s<T, TO, 1>(A, pitch, L, kz - L.N[2], out, accumulate, sc);
    else scatter_plane_s<T, TO, 0>(A, pitch, L, kz, out, accumulate, sc);
}

// Rows of `cols` points walked as point pairs: warp w takes rows w, w + nwarps,
// ...; its lanes take consecutive pairs of the row.  f(r, c), c even.
template <class F>
__device__ __forceinline__ void for_row_pairs(int rows, int cols, F &&f)
{
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int np = cols >> 1;
    for (int r = threadIdx.x >> 5; r < rows; r += nw)
        for (int j = lane; j < np; j += 32) f(r, 2 * j);
}

// a dense global plane of `cols`-point rows can move as point pairs when cols
// is even and the plane starts on a pair (the scratch planes do)
template <class T>
__device__ __forceinline__ bool pair_rows(int cols, const T *g)
{
    return !(cols & 1) && !(reinterpret_cast<uintptr_t>(g) & (2 * sizeof(T) - 1));
}

template <class T>
__device__ __forceinline__ void zero_region(T *A, int rows, int pitch)
{
    // rows * pitch is even and A starts on a pair
    using V = typename Pair<T>::type;
    V *a = reinterpret_cast<V *>(A);
    V z;
    z.x = T(0);
    z.y = T(0);
    for (int i = threadIdx.x; i < (rows * pitch) >> 1; i += blockDim.x) a[i] = z;
}

template <class T>
__device__ __forceinline__ void store_plane(const T *A, int pitch, int rows, int cols, T *g)
{
    if (pair_rows(cols, g)) {
        using V = typename Pair<T>::type;
        for_row_pairs(rows, cols, [&](int r, int c) {
            *reinterpret_cast<V *>(g + (size_t)r * cols + c) = *reinterpret_cast<const V *>(A + r * pitch + c);
        });
        return;
    }
    RowCol q(cols);
    for (int i = threadIdx.x; i < rows * cols; i += blockDim.x, q.next()) g[i] = A[q.r * pitch + q.c];
}

template <class T>
__device__ __forceinline__ void load_plane(T *A, int pitch, int rows, int cols, const T *g)
{
    RowCol q(cols);
    for (int i = threadIdx.x; i < rows * cols; i += blockDim.x, q.next()) A[q.r * pitch + q.c] = g[i];
}

// Owner of work item `it` when the items are laid out in runs, one run per
// orbital (or density chunk): prefix[0..n] ascending, prefix[0] = 0,
// prefix[n] = total.  Returns the o with prefix[o] <= it < prefix[o+1] by a
// 32-way search, each lane probing one point per round (the table is small
// and read by every CTA, so the probes hit L1).  All 32 lanes of the warp
// must call it.
__device__ __forceinline__ int find_owner(const int *__restrict__ prefix, int n, int it)
{
    const int lane = threadIdx.x & 31;
    int lo = 0, hi = n;
    while (hi - lo > 1) {
        const int step = (hi - lo + 31) >> 5;
        const int idx = lo + lane * step;
        const bool le = idx < hi && __ldg(prefix + idx) <= it;
        const unsigned m = __ballot_sync(0xffffffffu, le);
        lo += (31 - __clz(m)) * step;
        hi = min(hi, lo + step);
    }
    return lo;
}

// Asynchronous element copy global -> shared (cp.async, 4 or 8 bytes) with
// zero fill: every thread queues all its copies of a tile before waiting once,
// instead of one dependent load/store pair per element.  When !valid nothing
// is read and the element is set to zero (src is still a valid address).
template <class T>
__device__ __forceinline__ void cp_async_elem(T *dst, const T *src, bool valid)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    const int n = valid ? (int)sizeof(T) : 0;
    if constexpr (sizeof(T) == 4)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// point-pair copy global -> shared (8 bytes FP32, 16 bytes FP64), both addresses on a pair
template <class T>
__device__ __forceinline__ void cp_async_pair(T *dst, const T *src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    if constexpr (sizeof(T) == 4)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}

// point-pair copy with zero fill: when !valid nothing is read (src must still be
// a valid address) and the pair is set to zero
template <class T>
__device__ __forceinline__ void cp_async_pair_z(T *dst, const T *src, bool valid)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    const int n = valid ? 2 * (int)sizeof(T) : 0;
    if constexpr (sizeof(T) == 4)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
}

// load_plane through cp.async (A in shared memory); the caller waits
template <class T>
__device__ __forceinline__ void load_plane_async(T *A, int pitch, int rows, int cols, const T *g)
{
    if (pair_rows(cols, g)) {
        for_row_pairs(rows, cols, [&](int r, int c) { cp_async_pair(A + r * pitch + c, g + (size_t)r * cols + c); });
        return;
    }
    RowCol q(cols);
    for (int i = threadIdx.x; i < rows * cols; i += blockDim.x, q.next())
        cp_async_elem(A + q.r * pitch + q.c, g + i, true);
}

// gather_plane through cp.async (no scaling, same element type); the caller
// waits.  Each coefficient is one queued copy to its slot of the plane.
template <class T, int S3>
__device__ __forceinline__ void gather_plane_async_s(T *A, int pitch, const LrDev &L, int i3, const T *psi)
{
    const int H1 = half_off(L.N[0]), H2 = half_off(L.N[1]);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (!S3) {
        const int a = L.plane_c[i3], b = L.plane_c[i3 + 1];
        for (int sg = a + warp; sg < b; sg += nw) {
            const int4 d = L.seg_c[sg];
            for (int t = lane; t < d.z; t += 32) cp_async_elem(A + d.y * pitch + d.x + t, psi + d.w + t, true);
        }
    }
    const T *pf = psi + L.nvctr_c;
    const int a = L.plane_f[i3], b = L.plane_f[i3 + 1];
    for (int sg = a + warp; sg < b; sg += nw) {
        const int4 d = L.seg_f[sg];
        for (int t = lane; t < d.z; t += 32) {
            const T *src = pf + 7 * (size_t)(d.w + t);
#pragma unroll
            for (int c = 1; c <= 7; ++c) {
                if (fs3(c) != S3) continue;
                cp_async_elem(A + (fs2(c) * H2 + d.y) * pitch + fs1(c) * H1 + d.x + t, src + c - 1, true);
            }
        }
    }
}

template <class T>
__device__ void gather_plane_async(T *A, int pitch, const LrDev &L, int kz, const T *psi)
{
    if (kz >= L.N[2]) gather_plane_async_s<T, 1>(A, pitch, L, kz - L.N[2], psi);
    else gather_plane_async_s<T, 0>(A, pitch, L, kz, psi);
}

template <class TI>
__device__ __forceinline__ const TI *in_ptr(const OrbDev &o, const TI *base)
{
    return o.in_ptr ? (const TI *)o.in_ptr : base + o.psi;
}
template <class TO>
__device__ __forceinline__ TO *out_ptr(const OrbDev &o, TO *base)
{
    return o.out_ptr ? (TO *)o.out_ptr : base + o.psi;
}

// Resident CTAs per SM the plane kernels are compiled for (plane_ctas_per_sm
// in wvlh_internal.h): FP32 CTAs of 1024, 512, 384, 256 or 128 threads at 64,
// 64, 56, 64, 64 registers; FP64 CTAs of 512, 256 or 128 threads at up to 128
// registers; the 384-thread FP64 and the persistent variants take what their
// registers need.
__host__ __device__ constexpr int plane_min_blocks(bool fp32, bool persist, int nt)
{
    return persist ? 1 : plane_ctas_per_sm(fp32, nt);
}

// ---------------------------------------------------------------------------
// CG vectors the preconditioner's plane kernels fold in (MODE_PRECOND): K1
// forms the search direction while it gathers it (dir 1: d = r, the first
// iteration; dir 2: d = beta d + r with beta = rrn / rr, in T), and
// writes d back; K3 accumulates <d | A d> of its plane, into one partial per
// plane (as <P | W> of the fine planes it holds, since analysis is the
// transpose of synthesis).  dir 0 / d null: plain gather / scatter.
template <class T> struct CgIo {
    T *d;
    const T *r;
    const double *rr, *rrn;
    int dir;
};

// The direction update on one gathered plane: A holds d (or zeros when
// first), R the residual r of the same positions at row pitch rpitch = G1
// (dense, so it fits in the transposed-plane buffer); every coefficient
// position of the plane gets v = r (first) or beta d + r, written back to d
// in global memory and into A scaled by D^-1/2.
template <class T, int S3>
__device__ __forceinline__ void cg_dir_plane_s(T *A, int pitch, const T *R, int rpitch, const LrDev &L, int i3,
                                               T *__restrict__ d, T beta, bool first, const T *sc)
{
    const int H1 = half_off(L.N[0]), H2 = half_off(L.N[1]);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (!S3) {
        const int a = L.plane_c[i3], b = L.plane_c[i3 + 1];
        for (int sg = a + warp; sg < b; sg += nw) {
            const int4 q = L.seg_c[sg];
            for (int t = lane; t < q.z; t += 32) {
                const int pa = q.y * pitch + q.x + t, pr = q.y * rpitch + q.x + t;
                const T v = first ? R[pr] : fma(beta, A[pa], R[pr]);
                d[q.w + t] = v;
                A[pa] = v * sc[0];
            }
        }
    }
    T *df = d + L.nvctr_c;
    const int a = L.plane_f[i3], b = L.plane_f[i3 + 1];
    for (int sg = a + warp; sg < b; sg += nw) {
        const int4 q = L.seg_f[sg];
        for (int t = lane; t < q.z; t += 32) {
            T *dst = df + 7 * (size_t)(q.w + t);
#pragma unroll
            for (int c = 1; c <= 7; ++c) {
                if (fs3(c) != S3) continue;
                const int pa = (fs2(c) * H2 + q.y) * pitch + fs1(c) * H1 + q.x + t;
                const int pr = (fs2(c) * H2 + q.y) * rpitch + fs1(c) * H1 + q.x + t;
                const T v = first ? R[pr] : fma(beta, A[pa], R[pr]);
                dst[c - 1] = v;
                A[pa] = v * sc[c];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// K1: compressed psi -> P = S_x S_y psi (not in MODE_LOCDEN) and
// Q = M_x M_y P (not in MODE_PRECOND) for one wavelet z-plane.
//
// Plane kernels (K1, K3) hold two plane buffers A and B in shared memory.
// When two planes do not fit (FP64 boxes above about 60^3 periodic / 45^3
// free), B lives in gtmp, a global slice of gstride elements per CTA, and the
// grid is one CTA per SM looping over the work items (PERSIST; the slice is
// indexed by blockIdx, so no two running CTAs share it).  Otherwise every CTA
// runs one item.
template <class T, class TI, bool ALLPER, int MODE>
__device__ __forceinline__ void k1_item(const LrDev *__restrict__ lrs, const OrbDev *__restrict__ orbs,
                                        const int *__restrict__ pre, int norb, const TI *__restrict__ psi,
                                        T *__restrict__ scratch, const double *__restrict__ cprec, int it, T *sc,
                                        T *bslice, const CgIo<T> &cg)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    constexpr int SEG = Seg<T>::v;
    {
        const int oi = find_owner(pre, norb, it);   // item = (orbital, wavelet plane kz)
        const int kz = it - pre[oi];
        const OrbDev o = orbs[oi];
        const LrDev L = lrs[o.lr];
        const Dims d(L, ALLPER);
        const int pitch = d.pitch();
        T *A = reinterpret_cast<T *>(smem_raw);
        T *B = bslice ? bslice : A + d.rows() * pitch;

        if (MODE == MODE_PRECOND && threadIdx.x < 8) sc[threadIdx.x] = (T)prec_scal(L, cprec[oi], threadIdx.x);
        zero_region(A, d.G2, pitch);
        __syncthreads();
        if (MODE == MODE_PRECOND && cg.dir && std::is_same<T, TI>::value) {
            // the CG direction, updated and scaled on the way in: d and r of
            // the plane arrive by cp.async (d into A, r into B at pitch G1,
            // which the transposed-plane buffer always holds)
            T *dv = cg.d + o.psi;
            const bool first = cg.dir == 1;
            const T beta = first ? T(0) : (T)(cg.rrn[oi] / cg.rr[oi]);
            if (!first) gather_plane_async<T>(A, pitch, L, kz, dv);
            // (B in a global slice: plain loads, cp.async writes shared memory only)
            if (bslice) gather_plane<T, T>(B, d.G1, L, kz, cg.r + o.psi, nullptr);
            else gather_plane_async<T>(B, d.G1, L, kz, cg.r + o.psi);
            cp_async_wait_all();
            __syncthreads();
            if (kz >= d.N3) cg_dir_plane_s<T, 1>(A, pitch, B, d.G1, L, kz - d.N3, dv, beta, first, sc);
            else cg_dir_plane_s<T, 0>(A, pitch, B, d.G1, L, kz, dv, beta, first, sc);
        } else if constexpr (std::is_same<T, TI>::value) {
            gather_plane_async<T>(A, pitch, L, kz, in_ptr(o, psi));
            cp_async_wait_all();
            if constexpr (MODE == MODE_PRECOND) {
                // D^-1/2 per component k = s1 + 2 s2 + 4 s3 of each plane position
                __syncthreads();
                const int s3 = kz >= d.N3 ? 4 : 0;
                RowCol q(d.G1);
                for (int i = threadIdx.x; i < d.G2 * d.G1; i += blockDim.x, q.next())
                    A[q.r * pitch + q.c] *= sc[(q.c >= d.H1 ? 1 : 0) + (q.r >= d.H2 ? 2 : 0) + s3];
            }
        } else {
            gather_plane<T, TI>(A, pitch, L, kz, in_ptr(o, psi), MODE == MODE_PRECOND ? sc : nullptr);
        }
        __syncthreads();
        const int pt = d.pitchT(d.G2), ptf = d.pitchT(d.F2);
        pass_syn<T, SEG, true>(A, B, xpose_geom(d.G2, pitch, pt), d.N1, d.H1, d.p1);   // S_x: G2 rows, G1 -> F1, into B^T
        __syncthreads();
        pass_syn<T, SEG, true>(B, A, xpose_geom(d.F1, pt, pitch), d.N2, d.H2, d.p2);   // S_y: F1 lines, G2 -> F2, into A
        __syncthreads();
        if (MODE != MODE_LOCDEN) store_plane(A, pitch, d.F2, d.F1, scratch + o.sP + (size_t)kz * d.F2 * d.F1);
        if (MODE == MODE_PRECOND) return;
        if (d.p1) pass_mf<T, SEG, 0, true>(A, B, xpose_geom(d.F2, pitch, ptf), d.F1, d.I1);   // M_x into B^T
        else pass_mf<T, SEG, 2, true>(A, B, xpose_geom(d.F2, pitch, ptf), d.F1, d.I1);
        __syncthreads();
        if (d.p2) pass_mf<T, SEG, 0, true>(B, A, xpose_geom(d.I1, ptf, pitch), d.F2, d.I2);   // M_y into A
        else pass_mf<T, SEG, 2, true>(B, A, xpose_geom(d.I1, ptf, pitch), d.F2, d.I2);
        __syncthreads();
        store_plane(A, pitch, d.I2, d.I1, scratch + o.sQ + (size_t)kz * d.I2 * d.I1);
    }
}

template <class T, class TI, bool ALLPER, int MODE, bool PERSIST, int NT>
__global__ void __launch_bounds__(NT, plane_min_blocks(sizeof(T) == 4, PERSIST, NT)) k1_plane_forward(const LrDev *__restrict__ lrs,
                                                                  const OrbDev *__restrict__ orbs,
                                                                  const int *__restrict__ pre, int norb,
                                                                  const TI *__restrict__ psi, T *__restrict__ scratch,
                                                                  const double *__restrict__ cprec, T *gtmp,
                                                                  long long gstride, const CgIo<T> cg)
{
    __shared__ T sc[8];
    if (!PERSIST) {
        k1_item<T, TI, ALLPER, MODE>(lrs, orbs, pre, norb, psi, scratch, cprec, blockIdx.x, sc, nullptr, cg);
        return;
    }
    const int nwork = pre[norb];
    for (int it = blockIdx.x; it < nwork; it += gridDim.x) {
        __syncthreads();  // the previous item is done with A, B and sc
        k1_item<T, TI, ALLPER, MODE>(lrs, orbs, pre, norb, psi, scratch, cprec, it, sc,
                                     gtmp + (size_t)blockIdx.x * gstride, cg);
    }
}

// ---------------------------------------------------------------------------
// Passes along the z-pencils of a TC-column tile (columns side by side, z
// points TC apart): FP32 as line pairs with packed FMAs (wvlh_pairs.cuh),
// FP64 one line per thread (FP64 has no packed FMA, and its pairs would
// double the registers a thread holds).
template <class T>
__device__ __forceinline__ void z_syn(const T *src, T *dst, int N, int per)
{
    if constexpr (sizeof(T) == 4) pass2_syn<kPairSeg>(src, dst, PairGeom{TC / 2, TC, TC}, N, N, per);
    else pass_syn<T, Seg<T>::v>(src, dst, LineGeom{TC, 1, TC, 1, TC}, N, N, per);
}
template <class T>
__device__ __forceinline__ void z_ana(const T *src, T *dst, int N, int per)
{
    if constexpr (sizeof(T) == 4) pass2_ana<kPairSeg>(src, dst, PairGeom{TC / 2, TC, TC}, N, N, per);
    else pass_ana<T, Seg<T>::v>(src, dst, LineGeom{TC, 1, TC, 1, TC}, N, N, per);
}
template <class T, int MODE>
__device__ __forceinline__ void z_mf(const T *src, T *dst, int Lin, int Lout)
{
    if constexpr (sizeof(T) == 4) pass2_mf<kPairSeg, MODE>(src, dst, PairGeom{TC / 2, TC, TC}, Lin, Lout);
    else pass_mf<T, Seg<T>::v, MODE>(src, dst, LineGeom{TC, 1, TC, 1, TC}, Lin, Lout);
}
template <class T, bool EN = true>
__device__ __forceinline__ void z_kin(const T *src, T *dst, int L, int per, double scale, double *e)
{
    if constexpr (sizeof(T) == 4)
        pass2_kin<kPairSeg, false, EN>(src, dst, PairGeom{TC / 2, TC, TC}, L, per, scale, 0.f, e);
    else pass_kin<T, Seg<T>::v, false, false, EN>(src, dst, LineGeom{TC, 1, TC, 1, TC}, L, per, scale, T(0), e);
}

// ---------------------------------------------------------------------------
// K2: z-pencil tiles, one kernel instance per chain (each half the code of a
// two-chain kernel, which eases instruction fetch).  CHAIN 0:
// Z1 = A_z Mt_z (V . M_z S_z Q) in place of Q, E_pot partial.  CHAIN 1:
// Z2 = A_z K_z S_z P, E_kin(z) partial.
// NT threads per CTA: 256, or for FP32 320 / 384, which give the passes over
// 80- and 96-point z lines (32 line pairs x 10 or 12 eight-point segments)
// one item per thread; resident CTAs per SM at 64 registers a thread.
__host__ __device__ constexpr int z_min_blocks(bool fp32, int nt) { return fp32 ? 65536 / (64 * nt) : 1; }

template <class T, class TV, bool ALLPER, int CHAIN, int NT = kZThreads>
__global__ void __launch_bounds__(NT, z_min_blocks(sizeof(T) == 4, NT)) k2_zpencil(const LrDev *__restrict__ lrs, const OrbDev *__restrict__ orbs,
                                                        const int *__restrict__ pre, int norb,
                                                        const TV *__restrict__ pot, T *__restrict__ scratch,
                                                        double *__restrict__ part_pot, double *__restrict__ part_kin,
                                                        int part_stride, const __grid_constant__ CUtensorMap tm_in,
                                                        const __grid_constant__ CUtensorMap tm_out, int tma)
{
    // dynamic shared memory only (A, B, then the reduction slots and the TMA
    // barrier), so that the tile buffer starts the block's shared window
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // item = (orbital, tile): chain 0 tiles the I1 x I2 plane of Q, chain 1
    // the F1 x F2 plane of P, row-major; pre is the chain's own prefix table
    // CHAIN 2: chain 1 without the energy (the preconditioner's operator)
    constexpr int chain = CHAIN == 2 ? 1 : CHAIN;
    constexpr bool EN = CHAIN != 2;
    const int oi = find_owner(pre, norb, blockIdx.x);
    const int jj = blockIdx.x - pre[oi];   // tile index, also the energy slot
    const OrbDev o = orbs[oi];
    const LrDev L = lrs[o.lr];
    const Dims d(L, ALLPER);
    const int ntx = chain == 0 ? (d.I1 + TX - 1) / TX : (d.F1 + TX - 1) / TX;
    const int ty = jj / ntx, tx = jj - ty * ntx;
    const int x0 = tx * TX, y0 = ty * TY;
    const int zl = max(d.G3, max(d.F3, d.I3));
    T *A = reinterpret_cast<T *>(smem_raw);
    T *B = A + zl * TC;
    double *red = reinterpret_cast<double *>(B + zl * TC);
    uint64_t *tma_bar = reinterpret_cast<uint64_t *>(red + 32);
    // TMA writes the tile only into a kZAlign-aligned buffer
    tma = tma && !(smem_addr(A) & (kZAlign - 1));
    const int W = chain == 0 ? d.I1 : d.F1;   // plane width/height of the data
    const int H = chain == 0 ? d.I2 : d.F2;
    T *g = scratch + (chain == 0 ? o.sQ : o.sP);
    T *gz = scratch + (chain == 0 ? o.sQ : o.sZ);
    const size_t plane = (size_t)W * H;
    // element loops: thread t owns tile column c = t % TC at z = t / TC + k ZS
    constexpr int ZS = NT / TC;
    const int col = threadIdx.x % TC, zs = threadIdx.x / TC;
    const int xc = x0 + (col % TX), yc = y0 + (col / TX);
    const bool inside = xc < W && yc < H;
    const size_t colofs = (size_t)yc * W + xc;

    // column pairs (x, x + 1) of one tile row move as point pairs when the
    // plane rows have even length (the scratch planes start on a pair)
    const bool pairs = pair_rows(W, g);
    constexpr int TP = TC / 2, ZP = NT / TP;
    const int pc = 2 * (threadIdx.x % TP), zp = threadIdx.x / TP;
    const int xp = x0 + (pc % TX), yp = y0 + (pc / TX);
    const bool pin = xp < W && yp < H;   // W even: x + 1 is inside too
    const size_t pofs = (size_t)yp * W + xp;

    // load the tile: TC columns x G3 z' rows, zero outside the plane
    if (tma) {
        // one box {32, 2, G3} of the batch's (x, y, z, orbital) scratch tensor
        if (threadIdx.x == 0) mbar_init(tma_bar, 1);
        __syncthreads();
        if (threadIdx.x == 0) {
            mbar_expect_tx(tma_bar, (unsigned)(TC * d.G3 * sizeof(T)));
            tma_load_4d(A, &tm_in, x0, y0, 0, oi, tma_bar);
        }
        const bool ok = mbar_wait_bounded(tma_bar, 0);
        if (!__syncthreads_and(ok)) {
            // the copy did not complete in time: poison this tile's energy
            // slot (the orbital's energies come out NaN), give the copy in
            // flight one more bounded wait and leave the tile
            if (threadIdx.x == 0) {
                if (part_kin)
                    (chain == 0 ? part_pot : part_kin)[(size_t)oi * part_stride + jj] = __longlong_as_double(-1LL);
                mbar_wait_bounded(tma_bar, 0);
            }
            return;
        }
    } else {
        if (pairs) {
            for (int z = zp; z < d.G3; z += ZP)
                cp_async_pair_z(A + z * TC + pc, pin ? g + (size_t)z * plane + pofs : g, pin);
        } else {
            for (int z = zs; z < d.G3; z += ZS)
                cp_async_elem(A + z * TC + col, inside ? g + (size_t)z * plane + colofs : g, inside);
        }
        cp_async_wait_all();
        __syncthreads();
    }
    double e = 0.0;
    z_syn<T>(A, B, d.N3, d.p3);                                   // S_z: G3 -> F3
    __syncthreads();
    if constexpr (chain == 0) {
        if (d.p3) z_mf<T, 0>(B, A, d.F3, d.I3);                   // M_z: F3 -> I3
        else z_mf<T, 2>(B, A, d.F3, d.I3);
        __syncthreads();
        // psir <- V psir, epot += V psir^2 (orbitals/potential.f90:1011-1031);
        // per-thread partial sum in T, one FP64 conversion per thread (which
        // z values a thread sums depends on the block size, so the energy's
        // rounding does too)
        const TV *V = o.pot_ptr ? (const TV *)o.pot_ptr : pot + o.pot;
        T ep = T(0);
        constexpr int U = 4;   // potential loads in flight per thread
        // thread t takes the column pair (x, x + 1) of pair index t % (TC/2) at
        // z = t / (TC/2) + k ZP; the potential comes as a point pair when the
        // rows are even and the buffer starts on a pair, else point by point.
        // The arithmetic, and so the energy's summation order, is the same
        // either way (it does not depend on where the potential lives).
        using VV = typename Pair<TV>::type;
        using P2 = typename Pair<T>::type;
        const bool vpair = pairs && pair_rows(W, V);
        const bool in0 = xp < W && yp < H, in1 = xp + 1 < W && yp < H;
        const TV *vp = V + pofs;
        for (int z0 = zp; z0 < d.I3; z0 += U * ZP) {
            VV v[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int z = z0 + u * ZP;
                v[u].x = TV(0);
                v[u].y = TV(0);
                if (z < d.I3) {
                    if (vpair) {
                        if (in0) v[u] = *reinterpret_cast<const VV *>(vp + (size_t)z * plane);
                    } else {
                        if (in0) v[u].x = vp[(size_t)z * plane];
                        if (in1) v[u].y = vp[(size_t)z * plane + 1];
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int z = z0 + u * ZP;
                if (z < d.I3) {
                    P2 *a = reinterpret_cast<P2 *>(A + z * TC + pc);
                    P2 r = *a;
                    const T w0 = (T)v[u].x * r.x, w1 = (T)v[u].y * r.y;
                    if (in0) ep = fma(w0, r.x, ep);
                    if (in1) ep = fma(w1, r.y, ep);
                    r.x = in0 ? w0 : T(0);
                    r.y = in1 ? w1 : T(0);
                    *a = r;
                }
            }
        }
        e += (double)ep;
        __syncthreads();
        if (d.p3) z_mf<T, 1>(A, B, d.I3, d.F3);                   // Mt_z: I3 -> F3
        else z_mf<T, 3>(A, B, d.I3, d.F3);
        __syncthreads();
        z_ana<T>(B, A, d.N3, d.p3);                               // A_z: F3 -> G3
    } else {
        const double scale = -0.5 / ((0.5 * L.hgrid[2]) * (0.5 * L.hgrid[2]));
        z_kin<T, EN>(B, A, d.F3, d.p3, scale, &e);                // K_z X
        __syncthreads();
        z_ana<T>(A, B, d.N3, d.p3);                               // A_z: F3 -> G3
        __syncthreads();
        T *t = A; A = B; B = t;                                   // result in A
    }
    if (tma) {
        // the result tile goes back as one box (columns past the plane's
        // edge are not written)
        fence_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) {
            tma_store_4d(&tm_out, x0, y0, 0, oi, A);
            tma_store_drain();
        }
    } else {
        __syncthreads();
        if (pairs) {
            using V = typename Pair<T>::type;
            if (pin)
                for (int z = zp; z < d.G3; z += ZP)
                    *reinterpret_cast<V *>(gz + (size_t)z * plane + pofs) =
                        *reinterpret_cast<const V *>(A + z * TC + pc);
        } else if (inside) {
            for (int z = zs; z < d.G3; z += ZS) gz[(size_t)z * plane + colofs] = A[z * TC + col];
        }
    }
    if constexpr (EN) {
        const double s = block_sum(e, red);
        if (threadIdx.x == 0 && part_kin)
            (chain == 0 ? part_pot : part_kin)[(size_t)oi * part_stride + jj] = s;
    }
}

// ---------------------------------------------------------------------------
// K3 (MODE_LOCHAM): Hpsi plane kz = A_x A_y [Mt_x Mt_y Z1 + Z2 + (K_x + K_y) P]
// K3 (MODE_PRECOND): D^-1/2 A_x A_y [Z2 + c P + (K_x + K_y) P]
template <class T, class TO, bool ALLPER, int MODE>
__device__ __forceinline__ void k3_item(const LrDev *__restrict__ lrs, const OrbDev *__restrict__ orbs,
                                        const int *__restrict__ pre, int norb, const T *__restrict__ scratch,
                                        TO *__restrict__ hpsi, double *__restrict__ part_kin, int part_stride,
                                        int accumulate, const double *__restrict__ cprec, int it, T *sc,
                                        double *red, T *bslice, const TO *__restrict__ dotv)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    constexpr int SEG = Seg<T>::v;
    {
        const int oi = find_owner(pre, norb, it);   // item = (orbital, wavelet plane kz)
        const int kz = it - pre[oi];
        const OrbDev o = orbs[oi];
        const LrDev L = lrs[o.lr];
        const Dims d(L, ALLPER);
        const int pitch = d.pitch();
        T *A = reinterpret_cast<T *>(smem_raw);
        T *B = bslice ? bslice : A + d.rows() * pitch;

        T cshift = T(0);
        if (MODE == MODE_PRECOND) {
            cshift = (T)cprec[oi];
            if (threadIdx.x < 8) sc[threadIdx.x] = (T)prec_scal(L, cprec[oi], threadIdx.x);
        } else {
            load_plane_async(A, pitch, d.I2, d.I1, scratch + o.sQ + (size_t)kz * d.I2 * d.I1);
            cp_async_wait_all();
            __syncthreads();
            if (d.p1) pass_mf<T, SEG, 1, true>(A, B, xpose_geom(d.I2, pitch, d.pitchT(d.I2)), d.I1, d.F1);   // Mt_x into B^T
            else pass_mf<T, SEG, 3, true>(A, B, xpose_geom(d.I2, pitch, d.pitchT(d.I2)), d.I1, d.F1);
            __syncthreads();
            // Mt_y into A, plus Z2 (read from global memory as the outputs are stored)
            const T *z2 = scratch + o.sZ + (size_t)kz * d.F2 * d.F1;
            if (d.p2) pass_mf<T, SEG, 1, true, true>(B, A, xpose_geom(d.F1, d.pitchT(d.I2), pitch), d.I2, d.F2, z2, d.F1);
            else pass_mf<T, SEG, 3, true, true>(B, A, xpose_geom(d.F1, d.pitchT(d.I2), pitch), d.I2, d.F2, z2, d.F1);
            __syncthreads();
        }
        {
            const T *z2 = scratch + o.sZ + (size_t)kz * d.F2 * d.F1;
            const T *p = scratch + o.sP + (size_t)kz * d.F2 * d.F1;
            const int nf = d.F2 * d.F1;
            if (MODE != MODE_PRECOND && !bslice) {
                // P -> B (Z2 is already in A)
                load_plane_async(B, pitch, d.F2, d.F1, p);
                cp_async_wait_all();
            } else if (MODE == MODE_PRECOND && !bslice) {
                // P -> B and Z2 -> A asynchronously (the x kinetic pass adds c P)
                load_plane_async(B, pitch, d.F2, d.F1, p);
                load_plane_async(A, pitch, d.F2, d.F1, z2);
                cp_async_wait_all();
            } else {
                RowCol q(d.F1);
                for (int i = threadIdx.x; i < nf; i += blockDim.x, q.next()) {
                    const int e = q.r * pitch + q.c;
                    const T pv = p[i];
                    if (MODE == MODE_PRECOND) A[e] = z2[i];   // (MODE_LOCHAM: Z2 came with Mt_y)
                    B[e] = pv;
                }
            }
        }
        __syncthreads();
        // e: the kinetic energy partial (MODE_LOCHAM) or <d | A d> (MODE_PRECOND)
        // (the preconditioner's operator has no energy: its kinetic passes
        // are compiled without the energy terms, and its x pass adds c P)
        constexpr bool EN = MODE != MODE_PRECOND;
        double e = 0.0;
        const double sx = -0.5 / ((0.5 * L.hgrid[0]) * (0.5 * L.hgrid[0]));
        const double sy = -0.5 / ((0.5 * L.hgrid[1]) * (0.5 * L.hgrid[1]));
        pass_kin<T, SEG, true, true, EN, !EN>(B, A, rows_geom(d.F2, pitch), d.F1, d.p1, sx, cshift, &e);   // += K_x P
        __syncthreads();
        // += K_y P: the lines along y are the plane's columns, side by side
        // (F1 is even): FP32 takes them in pairs with packed FMAs
        if constexpr (sizeof(T) == 4) pass2_kin<kPairSeg, true, EN>(B, A, PairGeom{d.F1 / 2, pitch, pitch}, d.F2, d.p2, sy, 0.f, &e);
        else pass_kin<T, SEG, true, false, EN>(B, A, cols_geom(d.F1, pitch), d.F2, d.p2, sy, T(0), &e);
        __syncthreads();
        if (MODE == MODE_PRECOND && dotv) {
            // <d | A d> of this plane without reading d: analysis is the
            // transpose of synthesis, so <d, D^-1/2 A_x A_y W> = <P, W> with
            // P = S_x S_y D^-1/2 d (in B) and W the fine plane now in A
            RowCol q(d.F1);
            for (int i = threadIdx.x; i < d.F2 * d.F1; i += blockDim.x, q.next()) {
                const int el = q.r * pitch + q.c;
                e = fma((double)B[el], (double)A[el], e);
            }
            __syncthreads();   // A_x overwrites B
        }
        pass_ana<T, SEG, true>(A, B, xpose_geom(d.F2, pitch, d.pitchT(d.F2)), d.N1, d.H1, d.p1);   // A_x: F1 -> G1, into B^T
        __syncthreads();
        pass_ana<T, SEG, true>(B, A, xpose_geom(d.G1, d.pitchT(d.F2), pitch), d.N2, d.H2, d.p2);   // A_y: F2 -> G2, into A
        __syncthreads();
        scatter_plane<T, TO>(A, pitch, L, kz, out_ptr(o, hpsi), accumulate != 0, MODE == MODE_PRECOND ? sc : nullptr);
        const double s = block_sum(e, red);
        // slots 0 .. ntx1*nty1-1 belong to the z kernel's chain-1 tiles
        const int slot = ((d.F1 + TX - 1) / TX) * ((d.F2 + TY - 1) / TY) + kz;
        if (threadIdx.x == 0 && part_kin) part_kin[(size_t)oi * part_stride + slot] = s;
    }
}

// FP32: 3 CTAs per SM (56 registers), which the 75 KB of shared memory of a
// 96^2 plane pair allows; FP64 planes leave room for one CTA anyway
template <class T, class TO, bool ALLPER, int MODE, bool PERSIST, int NT>
__global__ void __launch_bounds__(NT, plane_min_blocks(sizeof(T) == 4, PERSIST, NT)) k3_plane_backward(const LrDev *__restrict__ lrs,
                                                                   const OrbDev *__restrict__ orbs,
                                                                   const int *__restrict__ pre, int norb,
                                                                   const T *__restrict__ scratch, TO *__restrict__ hpsi,
                                                                   double *__restrict__ part_kin, int part_stride,
                                                                   int accumulate, const double *__restrict__ cprec,
                                                                   T *gtmp, long long gstride,
                                                                   const TO *__restrict__ dotv)
{
    __shared__ double red[32];
    __shared__ T sc[8];
    if (!PERSIST) {
        k3_item<T, TO, ALLPER, MODE>(lrs, orbs, pre, norb, scratch, hpsi, part_kin, part_stride, accumulate, cprec,
                                     blockIdx.x, sc, red, nullptr, dotv);
        return;
    }
    const int nwork = pre[norb];
    for (int it = blockIdx.x; it < nwork; it += gridDim.x) {
        __syncthreads();  // the previous item is done with A, B, sc and red
        k3_item<T, TO, ALLPER, MODE>(lrs, orbs, pre, norb, scratch, hpsi, part_kin, part_stride, accumulate, cprec,
                                     it, sc, red, gtmp + (size_t)blockIdx.x * gstride, dotv);
    }
}

// fixed-order per-orbital sum of the energy partial slots
static __global__ void k_reduce_energies(const double *__restrict__ part_pot, const double *__restrict__ part_kin,
                                  int part_stride, int norb, double *__restrict__ ekin, double *__restrict__ epot)
{
    __shared__ double red[32];
    const int orb = blockIdx.x;
    if (orb >= norb) return;
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < part_stride; i += blockDim.x) {
        a += part_kin[(size_t)orb * part_stride + i];
        b += part_pot[(size_t)orb * part_stride + i];
    }
    const double sa = block_sum(a, red);
    __syncthreads();
    const double sb = block_sum(b, red);
    if (threadIdx.x == 0) {
        if (ekin) ekin[orb] = sa;
        if (epot) epot[orb] = sb;
    }
}

// ---------------------------------------------------------------------------
// Density z-kernel: for a tile of ISF columns, loop over the orbitals of one
// chunk: R = M_z S_z Q, acc += hfac R^2 (FP64), then write the chunk partial.
template <class T, bool ALLPER, int MAXP>
__global__ void __launch_bounds__(kZThreads) kd_density(const LrDev *__restrict__ lrs,
                                                        const OrbDev *__restrict__ orbs,
                                                        const int *__restrict__ pre, int nchunk,
                                                        const int *__restrict__ chunk_orb_start,
                                                        const int *__restrict__ chunk_orbs,
                                                        const long long *__restrict__ chunk_part,
                                                        const T *__restrict__ scratch, const double *__restrict__ hfac,
                                                        double *__restrict__ part)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // MAXP accumulators per thread: I3 * TC <= MAXP * kZThreads
    // item = (chunk, tile of the I1 x I2 plane, row-major)
    const int chunk = find_owner(pre, nchunk, blockIdx.x);
    const int j = blockIdx.x - pre[chunk];
    const int ob = chunk_orb_start[chunk], oe = chunk_orb_start[chunk + 1];
    const OrbDev o0 = orbs[chunk_orbs[ob]];
    const LrDev L = lrs[o0.lr];
    const Dims d(L, ALLPER);
    const int ntx = (d.I1 + TX - 1) / TX;
    const int x0 = (j % ntx) * TX, y0 = (j / ntx) * TY;
    const int zl = max(d.G3, max(d.F3, d.I3));
    T *A = reinterpret_cast<T *>(smem_raw);
    T *B = A + zl * TC;
    const int W = d.I1, H = d.I2;
    const size_t plane = (size_t)W * H;
    // thread t owns tile column c = t % TC at z = t / TC + k ZS
    constexpr int ZS = kZThreads / TC;
    const int col = threadIdx.x % TC, zs = threadIdx.x / TC;
    const int xc = x0 + (col % TX), yc = y0 + (col / TX);
    const bool inside = xc < W && yc < H;
    const size_t colofs = (size_t)yc * W + xc;
    double acc[MAXP];
#pragma unroll
    for (int k = 0; k < MAXP; ++k) acc[k] = 0.0;
    for (int oi = ob; oi < oe; ++oi) {
        const int orb = chunk_orbs[oi];
        const OrbDev o = orbs[orb];
        const T *g = scratch + o.sQ;
        __syncthreads();
        if (pair_rows(W, g)) {
            // column pairs as point pairs (even plane rows)
            constexpr int TP = TC / 2, ZP = kZThreads / TP;
            const int pc = 2 * (threadIdx.x % TP), zp = threadIdx.x / TP;
            const int xp = x0 + (pc % TX), yp = y0 + (pc / TX);
            const bool pin = xp < W && yp < H;
            const size_t pofs = (size_t)yp * W + xp;
            for (int z = zp; z < d.G3; z += ZP)
                cp_async_pair_z(A + z * TC + pc, pin ? g + (size_t)z * plane + pofs : g, pin);
        } else {
            for (int z = zs; z < d.G3; z += ZS)
                cp_async_elem(A + z * TC + col, inside ? g + (size_t)z * plane + colofs : g, inside);
        }
        cp_async_wait_all();
        __syncthreads();
        z_syn<T>(A, B, d.N3, d.p3);                               // S_z
        __syncthreads();
        if (d.p3) z_mf<T, 0>(B, A, d.F3, d.I3);                   // M_z
        else z_mf<T, 2>(B, A, d.F3, d.I3);
        __syncthreads();
        const double hf = hfac[orb];
#pragma unroll
        for (int k = 0; k < MAXP; ++k) {
            const int i = threadIdx.x + k * blockDim.x;
            if (i < d.I3 * TC) {
                const double r = (double)A[i];
                acc[k] = fma(hf * r, r, acc[k]);
            }
        }
    }
    double *out = part + chunk_part[chunk];
#pragma unroll
    for (int k = 0; k < MAXP; ++k) {
        const int i = threadIdx.x + k * blockDim.x;
        if (i < d.I3 * TC) {
            const int z = i / TC, c = i - z * TC;
            const int x = x0 + (c % TX), y = y0 + (c / TX);
            if (x < W && y < H) out[((size_t)z * H + y) * W + x] = acc[k];
        }
    }
}

// rho[group] += sum of the group's chunk partials, in chunk order
static __global__ void k_density_reduce(const int *__restrict__ group_chunk_start, const long long *__restrict__ group_rho,
                                 const int *__restrict__ group_n, const long long *__restrict__ chunk_part,
                                 const double *__restrict__ part, double *__restrict__ rho)
{
    const int g = blockIdx.y;
    const int n = group_n[g];
    const int cb = group_chunk_start[g], ce = group_chunk_start[g + 1];
    // packed batches: offsets into rho; orbital batches: addresses (rho null)
    double *r = rho ? rho + group_rho[g] : reinterpret_cast<double *>(group_rho[g]);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = r[i];
        for (int c = cb; c < ce; ++c) s += part[chunk_part[c] + i];
        r[i] = s;
    }
}

// ---------------------------------------------------------------------------
// Batched CG vector kernels (OpenCL/Preconditioner.c:130-195 with per-orbital
// scalars kept on the device).  Vectors are [psi_c | psi_f] per orbital at
// off[o], len[o] values; grid.y = orbital, grid.x = chunks of the vector.
// With VEC the values move 16 bytes per access (a scalar head up to the first
// 16-byte boundary of the orbital's range, then groups of 16 bytes, then a
// scalar tail); the launcher takes VEC when every vector of the call starts on
// a 16-byte boundary, so that all of them split alike.  Each thread's terms
// and the block sums come in a fixed order: the reductions are deterministic.
constexpr int kCgChunks = 16;

template <class T> struct alignas(16) Lanes {
    static constexpr int n = 16 / (int)sizeof(T);
    T v[n];
};
template <class T> __device__ __forceinline__ Lanes<T> ldv(const T *p) { return *reinterpret_cast<const Lanes<T> *>(p); }
template <class T> __device__ __forceinline__ void stv(T *p, const Lanes<T> &a) { *reinterpret_cast<Lanes<T> *>(p) = a; }

// e(i) for single values, g(i) for the 16-byte group starting at value i
template <class T, bool VEC, class E1, class EG>
__device__ __forceinline__ void cg_range(const T *p, int n, E1 &&e, EG &&g)
{
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
    if constexpr (!VEC) {
        for (int i = tid; i < n; i += nt) e(i);
    } else {
        constexpr int E = Lanes<T>::n;
        const int mis = (int)((reinterpret_cast<uintptr_t>(p) / sizeof(T)) % E);
        int head = mis ? E - mis : 0;
        head = head < n ? head : n;
        const int nv = (n - head) / E, t0 = head + nv * E;
        if (tid < head) e(tid);
        for (int j = tid; j < nv; j += nt) g(head + j * E);
        for (int i = t0 + tid; i < n; i += nt) e(i);
    }
}

// out[o] = sum of its chunk partials (fixed order); optionally copy into hist
static __global__ void k_cg_sum(int norb, const double *__restrict__ part, double *__restrict__ out,
                         double *__restrict__ hist)
{
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= norb) return;
    double s = 0.0;
    for (int c = 0; c < kCgChunks; ++c) s += part[o * kCgChunks + c];
    out[o] = s;
    if (hist) hist[o] = s;
}

// r = b - A x and the chunk partials of <r|r> (the first direction d = r is
// formed by the next K1)
template <class T, bool VEC>
__global__ void k_cg_init(const long long *__restrict__ off, const int *__restrict__ len, const T *__restrict__ b,
                          const T *__restrict__ ax, T *__restrict__ r, double *__restrict__ part)
{
    __shared__ double red[32];
    const int o = blockIdx.y;
    const long long base = off[o];
    const T *bo = b + base, *ao = ax + base;
    T *ro = r + base;
    double s = 0.0;
    cg_range<T, VEC>(
        bo, len[o],
        [&](int i) {
            const T v = bo[i] - ao[i];
            ro[i] = v;
            s += (double)v * (double)v;
        },
        [&](int i) {
            Lanes<T> v = ldv(bo + i);
            const Lanes<T> a = ldv(ao + i);
#pragma unroll
            for (int k = 0; k < Lanes<T>::n; ++k) {
                v.v[k] -= a.v[k];
                s += (double)v.v[k] * (double)v.v[k];
            }
            stv(ro + i, v);
        });
    const double t = block_sum(s, red);
    if (threadIdx.x == 0) part[o * kCgChunks + blockIdx.x] = t;
}

// alpha = rr / dAd; x += alpha d, r -= alpha A d, and the chunk partials of
// the new <r|r>
template <class T, bool VEC>
__global__ void k_cg_step(const long long *__restrict__ off, const int *__restrict__ len,
                          const double *__restrict__ rr, const double *__restrict__ dad, T *__restrict__ x,
                          const T *__restrict__ d, T *__restrict__ r, const T *__restrict__ ad,
                          double *__restrict__ part)
{
    __shared__ double red[32];
    const int o = blockIdx.y;
    const long long base = off[o];
    T *xo = x + base, *ro = r + base;
    const T *dn = d + base, *ao = ad + base;
    const T alpha = (T)(rr[o] / dad[o]);
    double s = 0.0;
    cg_range<T, VEC>(
        xo, len[o],
        [&](int i) {
            xo[i] = fma(alpha, dn[i], xo[i]);
            const T v = fma(-alpha, ao[i], ro[i]);
            ro[i] = v;
            s += (double)v * (double)v;
        },
        [&](int i) {
            Lanes<T> xv = ldv(xo + i), rv = ldv(ro + i);
            const Lanes<T> dv = ldv(dn + i), av = ldv(ao + i);
#pragma unroll
            for (int k = 0; k < Lanes<T>::n; ++k) {
                xv.v[k] = fma(alpha, dv.v[k], xv.v[k]);
                rv.v[k] = fma(-alpha, av.v[k], rv.v[k]);
                s += (double)rv.v[k] * (double)rv.v[k];
            }
            stv(xo + i, xv);
            stv(ro + i, rv);
        });
    const double t = block_sum(s, red);
    if (threadIdx.x == 0) part[o * kCgChunks + blockIdx.x] = t;
}

static __global__ void k_copy_scalars(int n, const double *__restrict__ a, double *__restrict__ b)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = a[i];
}

// x *= D^-1/2 per component (scale_psi_d, OpenCL/Uncompress.c:596): value i
// is coarse below nvctr_c, else fine component 1 + (i - nvctr_c) % 7
template <class T, bool VEC>
__global__ void k_cg_scale(const LrDev *__restrict__ lrs, const OrbDev *__restrict__ orbs,
                           const long long *__restrict__ off, const int *__restrict__ len,
                           const double *__restrict__ cprec, T *__restrict__ x)
{
    const int o = blockIdx.y;
    const OrbDev ob = orbs[o];
    const LrDev L = lrs[ob.lr];
    T sc[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) sc[k] = (T)prec_scal(L, cprec[o], k);
    T *xo = x + off[o];
    const int nc = L.nvctr_c;
    auto comp = [&](int i) { return i < nc ? 0 : 1 + (i - nc) % 7; };
    cg_range<T, VEC>(
        xo, len[o], [&](int i) { xo[i] *= sc[comp(i)]; },
        [&](int i) {
            Lanes<T> v = ldv(xo + i);
            int k = comp(i);
#pragma unroll
            for (int j = 0; j < Lanes<T>::n; ++j) {
                v.v[j] *= sc[k];
                // the next value's component: coarse until nvctr_c, then 1..7 cyclically
                k = (i + j + 1 < nc) ? 0 : (k == 0 || k == 7 ? 1 : k + 1);
            }
            stv(xo + i, v);
        });
}

// ---------------------------------------------------------------------------
// host launchers

// Launch shape of the plane kernels: two shared-memory planes when they fit,
// else one shared plane + a global slice per CTA after the batch scratch.
struct PlaneCfg {
    size_t smem = 0;
    int grid = 0;
    int threads = kPlaneThreads;
    long long gstride = 0;
    bool global_b = false;
};

static PlaneCfg plane_cfg(const Plan &p, int fp, int nwork)
{
    int dev = 0, lim = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&lim, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    PlaneCfg c;
    c.global_b = p.smem13[fp] > (size_t)lim - 1024;
    c.smem = c.global_b ? (size_t)p.plane_elems * (fp ? 8 : 4) : p.smem13[fp];
    c.grid = c.global_b ? (nwork < nsm ? nwork : nsm) : nwork;
    c.gstride = c.global_b ? p.planeB_elems : 0;
    c.threads = c.global_b ? kPlaneThreads : p.plane_threads[fp];
    return c;
}

template <class T, class TI, bool ALLPER, int MODE>
static auto k1_for(const PlaneCfg &pc) -> decltype(&k1_plane_forward<T, TI, ALLPER, MODE, false, kPlaneThreads>)
{
    if (pc.global_b) return k1_plane_forward<T, TI, ALLPER, MODE, true, kPlaneThreads>;
    if constexpr (sizeof(T) == 4)
        if (pc.threads == 1024) return k1_plane_forward<T, TI, ALLPER, MODE, false, 1024>;
    if (pc.threads == 512) return k1_plane_forward<T, TI, ALLPER, MODE, false, 512>;
    if (pc.threads == 128) return k1_plane_forward<T, TI, ALLPER, MODE, false, 128>;
    if (pc.threads == 256) return k1_plane_forward<T, TI, ALLPER, MODE, false, 256>;
    return k1_plane_forward<T, TI, ALLPER, MODE, false, kPlaneThreads>;
}

template <class T, class TO, bool ALLPER, int MODE>
static auto k3_for(const PlaneCfg &pc) -> decltype(&k3_plane_backward<T, TO, ALLPER, MODE, false, kPlaneThreads>)
{
    if (pc.global_b) return k3_plane_backward<T, TO, ALLPER, MODE, true, kPlaneThreads>;
    if constexpr (sizeof(T) == 4)
        if (pc.threads == 1024) return k3_plane_backward<T, TO, ALLPER, MODE, false, 1024>;
    if (pc.threads == 512) return k3_plane_backward<T, TO, ALLPER, MODE, false, 512>;
    if (pc.threads == 128) return k3_plane_backward<T, TO, ALLPER, MODE, false, 128>;
    if (pc.threads == 256) return k3_plane_backward<T, TO, ALLPER, MODE, false, 256>;
    return k3_plane_backward<T, TO, ALLPER, MODE, false, kPlaneThreads>;
}

// TMA maps of the z kernel's tiles: when every orbital of the batch lies in
// one region, the scratch planes of all orbitals form regular 4-D tensors
// (x, y, z, orbital) for Q (chain 0, read and written in place), P (chain 1
// input) and Z2 (chain 1 output); otherwise (several regions, or rows whose
// byte length TMA cannot stride) the tiles move with cp.async.
struct ZMaps {
    CUtensorMap q, p, z;
    int ok = 0;
};
template <class T>
static void zmaps(const Plan &p, T *scratch, ZMaps &m)
{
    memset(&m, 0, sizeof(m));
    if (p.orb_scratch <= 0) return;
    const int es = (int)sizeof(T);
    const long long G3 = p.tile_dims[0], F1 = p.tile_dims[1], F2 = p.tile_dims[2], I1 = p.tile_dims[3],
                    I2 = p.tile_dims[4];
    const long long sQ0 = G3 * F2 * F1, sZ0 = sQ0 + G3 * I2 * I1;
    m.ok = encode_tile_map(&m.q, scratch + sQ0, es, I1, I2, G3, p.norb, p.orb_scratch) &&
           encode_tile_map(&m.p, scratch, es, F1, F2, G3, p.norb, p.orb_scratch) &&
           encode_tile_map(&m.z, scratch + sZ0, es, F1, F2, G3, p.norb, p.orb_scratch);
}

// K1 / K3 launch with the plane configuration of the batch
template <class T, class TI, bool ALLPER, int MODE>
static cudaError_t run_k1(const Plan &p, const PlaneCfg &pc, const TI *psi, T *scratch, const double *cprec, T *gtmp,
                          cudaStream_t st, CgIo<T> cg = CgIo<T>{nullptr, nullptr, nullptr, nullptr, 0})
{
    cudaError_t err;
    auto k = k1_for<T, TI, ALLPER, MODE>(pc);
    if ((err = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pc.smem))) return err;
    k<<<pc.grid, pc.threads, pc.smem, st>>>(p.d_lr, p.d_orb, p.d_pre13, p.norb, psi, scratch, cprec, gtmp, pc.gstride,
                                            cg);
    return cudaSuccess;
}

template <class T, class TO, bool ALLPER, int MODE>
static cudaError_t run_k3(const Plan &p, const PlaneCfg &pc, const T *scratch, TO *out, double *part_kin,
                          int part_stride, int accumulate, const double *cprec, T *gtmp, cudaStream_t st,
                          const TO *dotv = nullptr)
{
    cudaError_t err;
    auto k = k3_for<T, TO, ALLPER, MODE>(pc);
    if ((err = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pc.smem))) return err;
    k<<<pc.grid, pc.threads, pc.smem, st>>>(p.d_lr, p.d_orb, p.d_pre13, p.norb, scratch, out, part_kin, part_stride,
                                            accumulate, cprec, gtmp, pc.gstride, dotv);
    return cudaSuccess;
}

// K2 launch with the block size zt (FP32: 256, 320 or 384; FP64: 256)
template <class T, class TV, bool ALLPER, int CHAIN>
static cudaError_t run_k2(int zt, int nwork, size_t sm2, const Plan &p, const int *pre, const TV *pot, T *scratch,
                          double *part_pot, double *part_kin, int part_stride, const CUtensorMap &m_in,
                          const CUtensorMap &m_out, int tma, cudaStream_t st)
{
    auto k = k2_zpencil<T, TV, ALLPER, CHAIN, kZThreads>;
    if constexpr (sizeof(T) == 4) {
        if (zt == 320) k = k2_zpencil<T, TV, ALLPER, CHAIN, 320>;
        else if (zt == 384) k = k2_zpencil<T, TV, ALLPER, CHAIN, 384>;
        else zt = kZThreads;
    } else {
        zt = kZThreads;
    }
    cudaError_t err;
    if ((err = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2))) return err;
    k<<<nwork, zt, sm2, st>>>(p.d_lr, p.d_orb, pre, p.norb, pot, scratch, part_pot, part_kin, part_stride, m_in,
                              m_out, tma);
    return cudaSuccess;
}

#ifdef WVLH_FUSED_COMMON
long long plane_tmp_elems(const Plan &p, int fp)
{
    int dev = 0, lim = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&lim, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    return p.smem13[fp] > (size_t)lim - 1024 ? (long long)nsm * p.planeB_elems : 0;
}
#endif
template <class T, class TIO, bool ALLPER>
static cudaError_t launch_locham_bc(const Plan &p, const TIO *psi, const TIO *pot, TIO *hpsi, T *scratch,
                                    double *part_pot, double *part_kin, double *ekin, double *epot, int accumulate,
                                    cudaStream_t st, cudaEvent_t *ev)
{
    const int fp = sizeof(T) == 8 ? 1 : 0;
    const PlaneCfg pc = plane_cfg(p, fp, p.n_work13);
    const size_t sm2 = p.smem2[fp] + kZExtra;
    T *gtmp = pc.global_b ? scratch + p.scratch_elems : nullptr;
    cudaError_t err;
    cudaMemsetAsync(part_pot, 0, sizeof(double) * (size_t)p.norb * p.part_stride, st);
    cudaMemsetAsync(part_kin, 0, sizeof(double) * (size_t)p.norb * p.part_stride, st);
    ZMaps zm;
    zmaps(p, scratch, zm);
    // optional per-kernel timing: ev[0..4] bracket K1, K2, K3 and the reduction
    if (ev) cudaEventRecord(ev[0], st);
    if ((err = run_k1<T, TIO, ALLPER, MODE_LOCHAM>(p, pc, psi, scratch, nullptr, gtmp, st))) return err;
    if (ev) cudaEventRecord(ev[1], st);
    if ((err = run_k2<T, TIO, ALLPER, 0>(p.z_threads[fp], p.n_work2, sm2, p, p.d_pre2, pot, scratch, part_pot,
                                         part_kin, p.part_stride, zm.q, zm.q, zm.ok, st)) ||
        (err = run_k2<T, TIO, ALLPER, 1>(p.z_threads[fp], p.n_work2p, sm2, p, p.d_pre2p, pot, scratch, part_pot,
                                         part_kin, p.part_stride, zm.p, zm.z, zm.ok, st)))
        return err;
    if (ev) cudaEventRecord(ev[2], st);
    if ((err = run_k3<T, TIO, ALLPER, MODE_LOCHAM>(p, pc, scratch, hpsi, part_kin, p.part_stride, accumulate, nullptr,
                                                   gtmp, st)))
        return err;
    if (ev) cudaEventRecord(ev[3], st);
    k_reduce_energies<<<p.norb, 128, 0, st>>>(part_pot, part_kin, p.part_stride, p.norb, ekin, epot);
    if (ev) cudaEventRecord(ev[4], st);
    return cudaGetLastError();
}

template <class T, class TIO>
cudaError_t launch_locham(const Plan &p, const TIO *psi, const TIO *pot, TIO *hpsi, T *scratch, double *part_pot,
                          double *part_kin, double *ekin, double *epot, int accumulate, cudaStream_t st,
                          cudaEvent_t *ev)
{
    if (p.all_periodic)
        return launch_locham_bc<T, TIO, true>(p, psi, pot, hpsi, scratch, part_pot, part_kin, ekin, epot,
                                              accumulate, st, ev);
    return launch_locham_bc<T, TIO, false>(p, psi, pot, hpsi, scratch, part_pot, part_kin, ekin, epot, accumulate,
                                           st, ev);
}

#ifdef WVLH_FUSED_F32
template cudaError_t launch_locham<float, float>(const Plan &, const float *, const float *, float *, float *,
                                                 double *, double *, double *, double *, int, cudaStream_t,
                                                 cudaEvent_t *);
#endif
#ifdef WVLH_FUSED_F64
template cudaError_t launch_locham<double, double>(const Plan &, const double *, const double *, double *, double *,
                                                   double *, double *, double *, double *, int, cudaStream_t,
                                                   cudaEvent_t *);
#endif

template <class T, bool ALLPER>
static cudaError_t launch_locden_bc(const Plan &p, const T *psi, const double *hfac, double *rho, T *scratch,
                                    double *part, cudaStream_t st)
{
    const int fp = sizeof(T) == 8 ? 1 : 0;
    const PlaneCfg pc = plane_cfg(p, fp, p.n_work13);
    const size_t sm2 = p.smem2[fp] + kZExtra;
    T *gtmp = pc.global_b ? scratch + p.scratch_elems : nullptr;
    cudaError_t err;
    auto kd = p.den_acc > 32 ? kd_density<T, ALLPER, 48> : kd_density<T, ALLPER, 32>;
    if ((err = cudaFuncSetAttribute(kd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2))) return err;
    if ((err = run_k1<T, T, ALLPER, MODE_LOCDEN>(p, pc, psi, scratch, nullptr, gtmp, st))) return err;
    kd<<<p.n_workd, kZThreads, sm2, st>>>(p.d_lr, p.d_orb, p.d_pred, p.nchunk, p.d_chunk_orb_start, p.d_chunk_orbs,
                                          p.d_chunk_part, scratch, hfac, part);
    dim3 g((p.max_group_n + 255) / 256 < 4096 ? (p.max_group_n + 255) / 256 : 4096, p.ngroup);
    k_density_reduce<<<g, 256, 0, st>>>(p.d_group_chunk_start, p.d_group_rho, p.d_group_n, p.d_chunk_part, part,
                                        rho);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_locden(const Plan &p, const T *psi, const double *hfac, double *rho, T *scratch, double *part,
                          cudaStream_t st)
{
    if (p.all_periodic) return launch_locden_bc<T, true>(p, psi, hfac, rho, scratch, part, st);
    return launch_locden_bc<T, false>(p, psi, hfac, rho, scratch, part, st);
}
#ifdef WVLH_FUSED_F32
template cudaError_t launch_locden<float>(const Plan &, const float *, const double *, double *, float *, double *,
                                          cudaStream_t);
#endif
#ifdef WVLH_FUSED_F64
template cudaError_t launch_locden<double>(const Plan &, const double *, const double *, double *, double *,
                                           double *, cudaStream_t);
#endif

// preconditioner operator y = D^-1/2 A (c + T) S D^-1/2 x for every orbital;
// cg.dir: x is the CG direction, formed by K1 (see CgIo); dotpart: K3's
// partials of <x | y> per plane (zeroed here first), or null
template <class T, bool ALLPER>
static cudaError_t launch_prec_apply_bc(const Plan &p, const T *x, T *y, const double *cprec, T *scratch,
                                        cudaStream_t st, const CgIo<T> &cg, double *dotpart)
{
    const int fp = sizeof(T) == 8 ? 1 : 0;
    PlaneCfg pc = plane_cfg(p, fp, p.n_work13);
    if (!pc.global_b) pc.threads = p.plane_threads_pre[fp];
    const size_t sm2 = p.smem2[fp] + kZExtra;
    T *gtmp = pc.global_b ? scratch + p.scratch_elems : nullptr;
    cudaError_t err;
    if ((err = run_k1<T, T, ALLPER, MODE_PRECOND>(p, pc, x, scratch, cprec, gtmp, st, cg))) return err;
    ZMaps zm;
    zmaps(p, scratch, zm);
    if ((err = run_k2<T, T, ALLPER, 2>(p.z_threads_pre[fp], p.n_work2p, sm2, p, p.d_pre2p, (const T *)nullptr, scratch,
                                       nullptr, nullptr, 0, zm.p, zm.z, zm.ok, st)))
        return err;
    if (dotpart) cudaMemsetAsync(dotpart, 0, sizeof(double) * (size_t)p.norb * p.part_stride, st);
    if ((err = run_k3<T, T, ALLPER, MODE_PRECOND>(p, pc, scratch, y, dotpart, dotpart ? p.part_stride : 0, 0, cprec,
                                                  gtmp, st, dotpart ? x : nullptr)))
        return err;
    return cudaGetLastError();
}

// out[o] = the sum of orbital o's stride partial slots: one warp per
// orbital, lane l summing slots l, l + 32, ... then a fixed shuffle tree
// (deterministic)
static __global__ void k_cg_sum_slots(int norb, const double *__restrict__ part, int stride, double *__restrict__ out)
{
    const int o = blockIdx.x;
    if (o >= norb) return;
    double s = 0.0;
    for (int k = threadIdx.x; k < stride; k += 32) s += part[(size_t)o * stride + k];
    s = warp_sum(s);
    if (threadIdx.x == 0) out[o] = s;
}

static bool aligned16(const void *p) { return !(reinterpret_cast<uintptr_t>(p) & 15); }

// The recurrence of Preconditioner.c:130-195 with two of its vector passes
// folded into the operator's kernels: K1 forms the direction
// d = r / d = beta d + r while gathering it, K3 accumulates <d | A d> while
// scattering A d.  Per iteration: apply (K1, K2, K3), alpha = rr / dAd, the
// x and r updates with the new <r|r> (k_cg_step), then rr <- rr_new once
// the next K1 has read both.
template <class T, bool VEC, class Apply>
static cudaError_t cg_loop(const Plan &p, int ncong, const double *cprec, T *x, const T *b, T *r, T *dvec, T *ad,
                           double *rr, double *dad, double *rrn, double *part, double *dotpart, double *hist,
                           Apply &&apply, cudaStream_t st)
{
    const dim3 vg(kCgChunks, p.norb);
    const int sg = (p.norb + 127) / 128;
    cudaError_t err;
    if ((err = apply(x, ad, CgIo<T>{nullptr, nullptr, nullptr, nullptr, 0}, nullptr))) return err;
    k_cg_init<T, VEC><<<vg, 256, 0, st>>>(p.d_orb_off, p.d_orb_len, b, ad, r, part);
    k_cg_sum<<<sg, 128, 0, st>>>(p.norb, part, rr, hist);
    for (int it = 0; it < ncong; ++it) {
        if ((err = apply(dvec, ad, CgIo<T>{dvec, r, rr, rrn, it == 0 ? 1 : 2}, dotpart))) return err;
        if (it > 0) k_copy_scalars<<<sg, 128, 0, st>>>(p.norb, rrn, rr);
        k_cg_sum_slots<<<p.norb, 32, 0, st>>>(p.norb, dotpart, p.part_stride, dad);
        k_cg_step<T, VEC><<<vg, 256, 0, st>>>(p.d_orb_off, p.d_orb_len, rr, dad, x, dvec, r, ad, part);
        k_cg_sum<<<sg, 128, 0, st>>>(p.norb, part, rrn, hist ? hist + (size_t)(it + 1) * p.norb : nullptr);
    }
    k_cg_scale<T, VEC><<<vg, 256, 0, st>>>(p.d_lr, p.d_orb, p.d_orb_off, p.d_orb_len, cprec, x);
    return cudaGetLastError();
}

// Batched CG of ocl_preconditioner_generic: x (in: initial guess, out:
// preconditioned), b right-hand side; work: r, d, ad vectors; scal:
// (5 + kCgChunks + part_stride) * norb doubles (scalars, chunk partials of
// the vector kernels, K3's per-plane partials of <d|Ad>); hist (optional):
// (ncong+1)*norb squared residual norms, entry 0 the initial one.
template <class T>
cudaError_t launch_precond(const Plan &p, int ncong, const double *cprec, T *x, const T *b, T *r, T *dvec, T *ad,
                           T *scratch, double *scal, double *hist, cudaStream_t st)
{
    double *rr = scal, *dad = scal + p.norb, *rrn = scal + 2 * p.norb, *part = scal + 5 * p.norb;
    double *dotpart = part + (size_t)kCgChunks * p.norb;
    auto apply = [&](const T *in, T *out, const CgIo<T> &cg, double *dp) {
        return p.all_periodic ? launch_prec_apply_bc<T, true>(p, in, out, cprec, scratch, st, cg, dp)
                              : launch_prec_apply_bc<T, false>(p, in, out, cprec, scratch, st, cg, dp);
    };
    const bool vec = aligned16(x) && aligned16(b) && aligned16(r) && aligned16(dvec) && aligned16(ad);
    return vec ? cg_loop<T, true>(p, ncong, cprec, x, b, r, dvec, ad, rr, dad, rrn, part, dotpart, hist, apply, st)
               : cg_loop<T, false>(p, ncong, cprec, x, b, r, dvec, ad, rr, dad, rrn, part, dotpart, hist, apply, st);
}
#ifdef WVLH_FUSED_F32
template cudaError_t launch_precond<float>(const Plan &, int, const double *, float *, const float *, float *, float *,
                                           float *, float *, double *, double *, cudaStream_t);
#endif
#ifdef WVLH_FUSED_F64
template cudaError_t launch_precond<double>(const Plan &, int, const double *, double *, const double *, double *,
                                            double *, double *, double *, double *, double *, cudaStream_t);
#endif

#ifdef WVLH_FUSED_COMMON
// FP32/FP64 FMA throughput probe: independent FMA chains held in registers.
template <class T>
__global__ void __launch_bounds__(256) k_fma_probe(T *out, int iters, T a, T b)
{
    T x[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) x[k] = T(threadIdx.x + k) * T(1e-3);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) x[k] = fma(x[k], a, b);
    }
    T s = T(0);
#pragma unroll
    for (int k = 0; k < 16; ++k) s += x[k];
    if (s == T(12345.678)) out[blockIdx.x] = s;  // keep the chains alive
}

cudaError_t fma_probe(int precision, int iters, float *ms, double *flops, cudaStream_t st)
{
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = nsm * 8;
    void *buf = nullptr;
    cudaError_t e = cudaMalloc(&buf, 8 * (size_t)blocks);
    if (e) return e;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    for (int rep = 0; rep < 2; ++rep) {  // first launch warms up
        cudaEventRecord(a, st);
        if (precision == 64) k_fma_probe<double><<<blocks, 256, 0, st>>>((double *)buf, iters, 0.999999, 1e-7);
        else k_fma_probe<float><<<blocks, 256, 0, st>>>((float *)buf, iters, 0.999999f, 1e-7f);
        cudaEventRecord(b, st);
    }
    cudaEventSynchronize(b);
    cudaEventElapsedTime(ms, a, b);
    *flops = 2.0 * 16.0 * (double)iters * 256.0 * blocks;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(buf);
    return cudaGetLastError();
}

#endif

}  // namespace wvlh
