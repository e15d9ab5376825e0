// Common device code of the wvlh library: filter constants, boundary helpers
// and the register-blocked 1D line passes every kernel is built from.
//
// A "line pass" applies one 1D operator of the Daubechies-16 local
// Hamiltonian (synthesis, analysis, magic filter, transposed magic filter,
// 29-tap kinetic) along lines of a shared-memory buffer.  Lines are addressed
// as base + line*ls + p*ps, so the same code walks rows, columns or z-pencils.
// Each thread owns a segment of SEG consecutive outputs of one line, loads
// the input window for the whole segment into registers once, and issues
// SEG*taps FMAs from registers; the filter taps are compile-time immediates.
//
// Operator definitions (the math of the reference, Fortran indices):
//  syn  (orbitals/convolut_simple_per.f90:89-103, free: OpenCL syngrow1d):
//       y(2i+o) = sum_{l=-4..4} ch(2l+o) s(i-l) + cg(2l+o) w(i-l)
//  ana  (convolut_simple_per.f90:11-57, free: OpenCL anashrink1d):
//       c(i) = sum_{l=-7..8} ch(l) y(2i+l),  d(i) = sum cg(l) y(2i+l)
//  mf   (convrot_n_per :200-243):  r(i) = sum_{l=-8..7} fil(l) x(i+l)
//  mft  (convrot_t_per :246-291):  x(i) = sum_{l=-7..8} fil(-l) r(i+l)
//  kin  (convolut_kinetic_per_T :377-460):
//       y(i) += -1/(2h^2) sum_{l=-14..14} a(|l|) x(i+l)
// Periodic lines wrap; free lines are zero outside and grow/shrink:
// fine grid f in [-7, 2N+6] (stored at q=f+7), ISF grid in [-14, 2N+14]
// (stored at r+14), exactly the OpenCL grow/shrink kernels' extents.
//
// FP32 energies: E_kin is accumulated in FP64 from the FP32 stencil result
// with the FP64 scale -1/(2h^2) and a low-order correction for the rounding of
// the six largest kinetic taps to FP32 (tap = hi + lo, lo applied to the
// already formed pair sums).  The synthesis and forward magic-filter passes,
// whose outputs feed E_kin and E_pot, start each FMA chain from the low-order
// parts of their largest taps, so the expectation of every rounded output
// carries the FP64 tap values.  Together these remove the systematic O(1e-8)
// relative bias that FP32-rounded constants put on the energies.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "wvl_filters.h"

namespace wvlh {

template <class T> struct Filt {
    static __device__ __forceinline__ constexpr T ch(int i) { return (T)(WVL_CH_AT(i)); }
    static __device__ __forceinline__ constexpr T cg(int i) { return (T)(WVL_CG_AT(i)); }
    static __device__ __forceinline__ constexpr T mf(int i) { return (T)(WVL_MF_AT(i)); }
    static __device__ __forceinline__ constexpr T kin(int i) { return (T)(WVL_KIN_AT(i)); }
    // residuals of the T-rounded taps (zero in FP64)
    static __device__ __forceinline__ constexpr T kin_lo(int i)
    {
        return (T)((WVL_KIN_AT(i)) - (double)(T)(WVL_KIN_AT(i)));
    }
    static __device__ __forceinline__ constexpr T ch_lo(int i) { return (T)((WVL_CH_AT(i)) - (double)(T)(WVL_CH_AT(i))); }
    static __device__ __forceinline__ constexpr T cg_lo(int i) { return (T)((WVL_CG_AT(i)) - (double)(T)(WVL_CG_AT(i))); }
    static __device__ __forceinline__ constexpr T mf_lo(int i) { return (T)((WVL_MF_AT(i)) - (double)(T)(WVL_MF_AT(i))); }
};

// taps whose FP32 rounding residual is carried (see the header comment)
__host__ __device__ constexpr bool big_tap(double v, double thr) { return v > thr || v < -thr; }

// FP32 passes whose outputs feed the energies (synthesis, forward magic
// filter) start each output's FMA chain from lo * x of their largest taps, lo
// = c - fl(c) the tap's FP32 rounding residual: the rounding of a tap biases
// every output the same way (relative ~1e-8 on the energies), and the bias of
// tap c goes as |lo(c) c|, so the few largest taps carry nearly all of it.
// Seeded: |c| > 0.1 for the Daubechies filters (four per output, 99.9 % of
// the bias) and the 0.994 centre tap of the magic filter (98 %).
constexpr double kSynSeedTap = 0.1;
constexpr double kMfSeedTap = 0.5;

// Fine-grid and ISF-grid extents of one dimension with N coarse cells.
__host__ __device__ __forceinline__ int fine_len(int N, int per) { return per ? 2 * N : 2 * N + 14; }
__host__ __device__ __forceinline__ int isf_len(int N, int per) { return per ? 2 * N : 2 * N + 29; }

// Periodic index for -L <= p < 3L, without a division.  The fused passes only
// see periodic lines of at least 8 coarse / 16 fine points, and their windows
// reach at most 15 points below and SEG + 13 (<= 21) points above the line.
__device__ __forceinline__ int wrap_near(int p, int L)
{
    p += p < 0 ? L : 0;
    p -= p >= L ? L : 0;
    p -= p >= L ? L : 0;
    return p;
}

// Plane layout of the fused kernels' shared-memory buffers.  A coarse line is
// [s(0..N-1) | w(0..N-1)] with the wavelet half at the even offset
// half_off(N), so both halves start on a point pair.  Buffers whose lines run
// along rows use a row pitch with pitch % 4 == 2: every row starts on a point
// pair (8 bytes FP32, 16 bytes FP64), which lets the unit-stride passes load
// two points per instruction, and lanes that take consecutive rows still hit
// distinct banks (half-warp phases for 8-byte, quarter-warp for 16-byte).
__host__ __device__ constexpr int half_off(int N) { return (N + 1) & ~1; }
__host__ __device__ constexpr int coarse_width(int N) { return half_off(N) + N; }
__host__ __device__ constexpr int vec_pitch(int m) { return ((m + 1) & ~1) + ((((m + 1) & ~1) & 3) == 0 ? 2 : 0); }

template <class T> struct Pair;
template <> struct Pair<float> { using type = float2; };
template <> struct Pair<double> { using type = double2; };

// Load x[k] = line(p0 + k), k < W, with periodic wrap or zero padding; the
// common interior case takes a single base address and constant strides.
template <class T, int W>
__device__ __forceinline__ void load_window(T (&x)[W], const T *in, int ps, int p0, int L, int per)
{
    if (p0 >= 0 && p0 + W <= L) {
        const T *b = in + p0 * ps;
#pragma unroll
        for (int k = 0; k < W; ++k) x[k] = b[k * ps];
    } else if (per) {
#pragma unroll
        for (int k = 0; k < W; ++k) x[k] = in[wrap_near(p0 + k, L) * ps];
    } else {
#pragma unroll
        for (int k = 0; k < W; ++k) {
            const int p = p0 + k;
            x[k] = ((unsigned)p < (unsigned)L) ? in[p * ps] : T(0);
        }
    }
}

// Window load for a unit-stride line that starts on a point pair, q0 even:
// x[k] = line(q0 + SHIFT + k).  The window is read as W/2 + 1 point pairs from
// the pair boundary below q0 + SHIFT, never past the pair holding the line's
// last point: the rows hold at least L + 1 points when L is odd, so reads stay
// inside the row.  Zero padding (free lines) masks whole pairs and the point
// after an odd line's end; periodic wrap moves whole pairs when L is even.
// Periodic lines of odd length (coarse lines of an odd box) take the scalar
// path at the line ends.
template <class T, int W, int SHIFT>
__device__ __forceinline__ void load_window_u(T (&x)[W], const T *in, int q0, int L, int per)
{
    using V = typename Pair<T>::type;
    constexpr int R = SHIFT & 1;
    constexpr int A0 = SHIFT - R;
    constexpr int NV = (W + R + 1) / 2;
    const int a = q0 + A0;
    T y[2 * NV];
    if (a >= 0 && q0 + SHIFT + W <= L) {
        const V *b = reinterpret_cast<const V *>(in + a);
#pragma unroll
        for (int c = 0; c < NV; ++c) {
            const V v = b[c];
            y[2 * c] = v.x;
            y[2 * c + 1] = v.y;
        }
    } else if (!per) {
#pragma unroll
        for (int c = 0; c < NV; ++c) {
            const int p = a + 2 * c;
            V v;
            v.x = T(0);
            v.y = T(0);
            if ((unsigned)p < (unsigned)L) v = *reinterpret_cast<const V *>(in + p);
            y[2 * c] = v.x;
            y[2 * c + 1] = p + 1 < L ? v.y : T(0);
        }
    } else if (!(L & 1)) {
#pragma unroll
        for (int c = 0; c < NV; ++c) {
            const V v = *reinterpret_cast<const V *>(in + wrap_near(a + 2 * c, L));
            y[2 * c] = v.x;
            y[2 * c + 1] = v.y;
        }
    } else {
        load_window<T, W>(x, in, 1, q0 + SHIFT, L, per);
        return;
    }
#pragma unroll
    for (int k = 0; k < W; ++k) x[k] = y[k + R];
}

// UNIT passes read lines with unit stride from rows that start on a point pair
template <class T, int W, int SHIFT, bool UNIT>
__device__ __forceinline__ void load_window_g(T (&x)[W], const T *in, int ps, int q0, int L, int per)
{
    if constexpr (UNIT) load_window_u<T, W, SHIFT>(x, in, q0, L, per);
    else load_window<T, W>(x, in, ps, q0 + SHIFT, L, per);
}

// Distribute (line, segment) work items over the block: consecutive threads
// take consecutive lines so that x-passes (lanes = rows, odd pitch) and
// y/z-passes (lanes = contiguous columns) are both bank-conflict free.
template <class F>
__device__ __forceinline__ void for_items(int nlines, int nseg, F &&f)
{
    // item it = s * nlines + line, stepped by blockDim with one division per pass
    const int items = nlines * nseg;
    const int bd = blockDim.x;
    int s = threadIdx.x / nlines, line = threadIdx.x - s * nlines;
    const int ds = bd / nlines, dl = bd - ds * nlines;
    for (int it = threadIdx.x; it < items; it += bd) {
        f(line, s);
        line += dl;
        s += ds;
        if (line >= nlines) {
            line -= nlines;
            ++s;
        }
    }
}

// (row, col) of element i = row * cols + col for i = threadIdx.x + k * blockDim.x,
// advanced without a division per element
struct RowCol {
    int r, c, dr, dc, cols;
    __device__ __forceinline__ explicit RowCol(int cols_) : cols(cols_)
    {
        r = threadIdx.x / cols;
        c = threadIdx.x - r * cols;
        dr = blockDim.x / cols;
        dc = blockDim.x - dr * cols;
    }
    __device__ __forceinline__ void next()
    {
        c += dc;
        r += dr;
        if (c >= cols) {
            c -= cols;
            ++r;
        }
    }
};

// for_items over a pass body instantiated twice: FULL = true for segments
// whose outputs all fall inside the line (no per-output bounds test), false
// for the clipped ones; full(line, s) tells which.
template <class Full, class Body>
__device__ __forceinline__ void for_items2(int nlines, int nseg, Full &&full, Body &&body)
{
    for_items(nlines, nseg, [&](int line, int s) {
        if (full(s)) body(line, s, std::true_type{});
        else body(line, s, std::false_type{});
    });
}

struct LineGeom {
    int nlines;
    int src_ls, src_ps;
    int dst_ls, dst_ps;
};

// ---------------------------------------------------------------- synthesis
// src line: [s(0..N-1) | w(0..N-1)], the wavelet half at offset H (N, or
// half_off(N) in the fused planes); dst line: F = fine_len(N,per) values.
template <class T, int SEG, bool UNIT = false>
__device__ __forceinline__ void pass_syn(const T *src, T *dst, const LineGeom g, int N, int H, int per)
{
    static_assert(SEG % 2 == 0, "even segment");
    constexpr int W = SEG / 2 + 8;
    const int F = fine_len(N, per);
    const int off = per ? 0 : 7;      // storage index q = f + off
    const int fstart = per ? 0 : -8;  // even start in Fortran fine coordinates
    const int nseg = (F + off - fstart + SEG - 1) / SEG;
    auto full = [&](int s) {
        const int q0 = fstart + s * SEG + off;
        return q0 >= 0 && q0 + SEG <= F;
    };
    for_items2(g.nlines, nseg, full, [&](int line, int s, auto full_t) {
        constexpr bool FULL = decltype(full_t)::value;
        const T *in = src + line * g.src_ls;
        T *out = dst + line * g.dst_ls;
        const int f0 = fstart + s * SEG;
        const int c0 = f0 / 2;  // f0 is even, so f0/2 is exact (and even)
        T xs[W], xw[W];
        load_window_g<T, W, -4, UNIT>(xs, in, g.src_ps, c0, N, per);
        load_window_g<T, W, -4, UNIT>(xw, in + H * g.src_ps, g.src_ps, c0, N, per);
#pragma unroll
        for (int t = 0; t < SEG; ++t) {
            const int q = f0 + t + off;
            const int o = t & 1;
            const int ic = t / 2 + 4;  // window index of coarse position i0 + t/2
            T acc = T(0);
            if constexpr (sizeof(T) == 4) {
                // low-order parts of the largest taps seed the FMA chain
#pragma unroll
                for (int l = -4; l <= 4; ++l) {
                    const int m = 2 * l + o;
                    if (m < -7 || m > 8) continue;
                    if (big_tap(WVL_CH_AT(m + 7), kSynSeedTap)) acc = fma(Filt<T>::ch_lo(m + 7), xs[ic - l], acc);
                    if (big_tap(WVL_CG_AT(m + 7), kSynSeedTap)) acc = fma(Filt<T>::cg_lo(m + 7), xw[ic - l], acc);
                }
            }
#pragma unroll
            for (int l = -4; l <= 4; ++l) {
                const int m = 2 * l + o;  // ch_syn(m) = ch(m) for m in [-7,8]
                if (m < -7 || m > 8) continue;
                acc = fma(Filt<T>::ch(m + 7), xs[ic - l], acc);
                acc = fma(Filt<T>::cg(m + 7), xw[ic - l], acc);
            }
            if (FULL || (unsigned)q < (unsigned)F) out[q * g.dst_ps] = acc;
        }
    });
}

// ---------------------------------------------------------------- analysis
// src line: F fine values; dst line: [c(0..N-1) | d(0..N-1)], d at offset H
template <class T, int SEG, bool UNIT = false>
__device__ __forceinline__ void pass_ana(const T *src, T *dst, const LineGeom g, int N, int H, int per)
{
    static_assert(SEG % 2 == 0, "even segment");
    constexpr int HS = SEG / 2;
    constexpr int W = SEG + 14;
    const int F = fine_len(N, per);
    const int nseg = (N + HS - 1) / HS;
    auto full = [&](int s) { return s * HS + HS <= N; };
    for_items2(g.nlines, nseg, full, [&](int line, int s, auto full_t) {
        constexpr bool FULL = decltype(full_t)::value;
        const T *in = src + line * g.src_ls;
        T *out = dst + line * g.dst_ls;
        const int i0 = s * HS;
        T x[W];
        if (per) load_window_g<T, W, -7, UNIT>(x, in, g.src_ps, 2 * i0, F, 1);
        else load_window_g<T, W, 0, UNIT>(x, in, g.src_ps, 2 * i0, F, 0);
#pragma unroll
        for (int t = 0; t < HS; ++t) {
            T ci = T(0), di = T(0);
#pragma unroll
            for (int l = 0; l < 16; ++l) {
                ci = fma(Filt<T>::ch(l), x[2 * t + l], ci);
                di = fma(Filt<T>::cg(l), x[2 * t + l], di);
            }
            const int i = i0 + t;
            if (FULL || i < N) {
                out[i * g.dst_ps] = ci;
                out[(i + H) * g.dst_ps] = di;
            }
        }
    });
}

// ---------------------------------------------------------------- magic filter
// MODE 0: mf periodic, 1: mft periodic, 2: mf grow (F -> F+15), 3: mft shrink (F+15 -> F)
// ADDG: every output also gains addg[line + q * addg_ps] (a plane in global
// memory, read as the outputs are stored)
template <class T, int SEG, int MODE, bool UNIT = false, bool ADDG = false>
__device__ __forceinline__ void pass_mf(const T *src, T *dst, const LineGeom g, int Lin, int Lout,
                                        const T *__restrict__ addg = nullptr, int addg_ps = 0)
{
    constexpr int W = SEG + 15;
    constexpr int shift = MODE == 0 ? -8 : MODE == 1 ? -7 : MODE == 2 ? -15 : 0;
    constexpr bool rev = (MODE == 1 || MODE == 3);
    constexpr int per = (MODE <= 1);
    const int nseg = (Lout + SEG - 1) / SEG;
    auto full = [&](int s) { return s * SEG + SEG <= Lout; };
    for_items2(g.nlines, nseg, full, [&](int line, int s, auto full_t) {
        constexpr bool FULL = decltype(full_t)::value;
        const T *in = src + line * g.src_ls;
        T *out = dst + line * g.dst_ls;
        const int q0 = s * SEG;
        T x[W];
        load_window_g<T, W, shift, UNIT>(x, in, g.src_ps, q0, Lin, per);
#pragma unroll
        for (int t = 0; t < SEG; ++t) {
            T acc = T(0);
            if constexpr (sizeof(T) == 4 && !rev) {
                // forward magic filter feeds E_pot: seed with the residual of
                // its centre tap
#pragma unroll
                for (int k = 0; k < 16; ++k)
                    if (big_tap(WVL_MF_AT(k), kMfSeedTap)) acc = fma(Filt<T>::mf_lo(k), x[t + k], acc);
            }
#pragma unroll
            for (int k = 0; k < 16; ++k) acc = fma(Filt<T>::mf(rev ? 15 - k : k), x[t + k], acc);
            const int q = q0 + t;
            if (FULL || q < Lout) {
                if constexpr (ADDG) acc += addg[line + q * addg_ps];
                out[q * g.dst_ps] = acc;
            }
        }
    });
}

// ---------------------------------------------------------------- kinetic
// dst(q) = (ACC ? dst(q) : cshift * src(q)) + scale * sum_l a(|l|) src(q+l)
// with scale = -1/(2h^2) (cshift: the preconditioner's c of (T + c),
// OpenCL/Preconditioner.c:108); ekin += src(q) * scale * conv in FP64.
// UNIT: source and destination lines are unit-stride rows starting on a point
// pair (window and full output segments move as point pairs).  EN: compute
// the energy (else ekin is left alone); ACCS (with ACC): dst(q) also gains
// cshift src(q).
template <class T, int SEG, bool ACC, bool UNIT = false, bool EN = true, bool ACCS = false>
__device__ __forceinline__ void pass_kin(const T *src, T *dst, const LineGeom g, int L, int per, double scale_d, T cshift,
                         double *ekin)
{
    constexpr int W = SEG + 28;
    const T scale = (T)scale_d;
    const int nseg = (L + SEG - 1) / SEG;
    double e = 0.0;
    auto full = [&](int s) { return s * SEG + SEG <= L; };
    for_items2(g.nlines, nseg, full, [&](int line, int s, auto full_t) {
        constexpr bool FULL = decltype(full_t)::value;
        const T *in = src + line * g.src_ls;
        T *out = dst + line * g.dst_ls;
        const int q0 = s * SEG;
        T x[W];
        load_window_g<T, W, -14, UNIT>(x, in, g.src_ps, q0, L, per);
        // per-segment partial sums of x.conv, converted to FP64 once per
        // segment (the rounding of these short sums is unbiased); in FP32 the
        // taps' rounding residuals lo(l) enter E_kin through the lag sums
        // C(l) = sum_q x(q) x(q-l) of the three largest taps, lo(0) C(0) +
        // 2 sum lo(l) C(l), which over whole lines equals the per-output
        // correction (as the line-pair kinetic pass does)
        T es = T(0);
        [[maybe_unused]] T c0 = T(0), c1 = T(0), c2 = T(0);
        T prev = T(0);
#pragma unroll
        for (int t = 0; t < SEG; ++t) {
            T conv = Filt<T>::kin(0) * x[t + 14];
#pragma unroll
            for (int l = 1; l <= 14; ++l) {
                const T pr = x[t + 14 + l] + x[t + 14 - l];
                conv = fma(Filt<T>::kin(l), pr, conv);
            }
            const int q = q0 + t;
            if (EN && (FULL || q < L)) {
                es = fma(x[t + 14], conv, es);
                if constexpr (sizeof(T) == 4) {
                    c0 = fma(x[t + 14], x[t + 14], c0);
                    c1 = fma(x[t + 14], x[t + 13], c1);
                    c2 = fma(x[t + 14], x[t + 12], c2);
                }
            }
            // unit-stride rows store each point pair once both are formed (a
            // clipped segment of an even line ends on a whole pair)
            if (UNIT && (FULL || !(L & 1))) {
                if (FULL || q < L) {
                    if (t & 1) {
                        using V = typename Pair<T>::type;
                        V *o = reinterpret_cast<V *>(out + q - 1);
                        V v;
                        if (ACC) {
                            v = *o;
                            if (ACCS) {
                                v.x = fma(cshift, x[t + 13], v.x);
                                v.y = fma(cshift, x[t + 14], v.y);
                            }
                        } else {
                            v.x = cshift * x[t + 13];
                            v.y = cshift * x[t + 14];
                        }
                        v.x = fma(scale, prev, v.x);
                        v.y = fma(scale, conv, v.y);
                        *o = v;
                    } else {
                        prev = conv;
                    }
                }
            } else if (FULL || q < L) {
                const T base = ACC ? (ACCS ? fma(cshift, x[t + 14], out[q * g.dst_ps]) : out[q * g.dst_ps])
                                   : cshift * x[t + 14];
                out[q * g.dst_ps] = fma(scale, conv, base);
            }
        }
        if constexpr (EN) {
            double el = 0.0;
            if constexpr (sizeof(T) == 4)
                el = (double)Filt<T>::kin_lo(0) * (double)c0 +
                     2.0 * ((double)Filt<T>::kin_lo(1) * (double)c1 + (double)Filt<T>::kin_lo(2) * (double)c2);
            e += ((double)es + el) * scale_d;
        }
    });
    if (EN && ekin) *ekin += e;
}

// ---------------------------------------------------------------- reductions
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// block-wide sum, result valid in thread 0; red must hold 32 doubles
__device__ __forceinline__ double block_sum(double v, double *red)
{
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (wid == 0) {
        r = (lane < (int)(blockDim.x >> 5)) ? red[lane] : 0.0;
        r = warp_sum(r);
    }
    return r;
}

}  // namespace wvlh
