// Line-pair forms of the 1D passes (FP32), for lines that lie side by side
// in shared memory: the z-pencils of the z kernel's tiles (lines are the
// tile's columns, points TC apart).  A thread takes two neighbouring lines at
// once: every window value is one 8-byte shared-memory load covering both
// lines, every output pair one 8-byte store, and every tap one packed
// fma.rn.f32x2 (__ffma2_rn) for the two lines.  Against one line per thread
// this halves the loads, stores and FMA instructions a thread issues; the FMA
// pipe still does the same work (a packed FMA occupies it for two cycles).
//
// FP32 accuracy.  Rounding a tap c to FP32 leaves a residual lo = c - fl(c),
// |lo| <= 2^-24 |c|, that biases every output the same way and so the
// energies (relative ~1e-8).  The synthesis and forward magic-filter passes,
// whose outputs feed E_kin and E_pot, start each output's FMA chain from
// lo * x of their largest taps (|c| > 0.1 for the Daubechies filters, the
// 0.994 centre tap of the magic filter): those carry over 99 % of the bias
// (the rest, below 2e-10 relative, is left), and as the first terms of the
// chain they survive in the expected value of the rounded output.  The
// kinetic pass corrects E_kin for its three largest taps through short-lag
// autocorrelations (pass2_kin).
#pragma once
#include <cuda_runtime.h>

#include "wvlh_common.cuh"

namespace wvlh {

template <class T> struct PV;
template <> struct PV<float> {
    using V = float2;
    static __device__ __forceinline__ V fma(float c, V x, V a) { return __ffma2_rn(make_float2(c, c), x, a); }
    static __device__ __forceinline__ V fmav(V c, V x, V a) { return __ffma2_rn(c, x, a); }
    static __device__ __forceinline__ V mul(float c, V x) { return __fmul2_rn(make_float2(c, c), x); }
    static __device__ __forceinline__ V zero() { return make_float2(0.f, 0.f); }
};

// the pair passes seed the taps kSynSeedTap / kMfSeedTap select
// (wvlh_common.cuh), as the one-line passes do
constexpr int kKinLags = 3;

// outputs per line of one thread's segment: eight outputs share a window of
// SEG + taps - 1 loads, which keeps the shared-memory bytes per output below
// what the FMA pipe consumes, with the window in registers
constexpr int kPairSeg = 8;

// npairs line pairs: pair lp holds lines 2 lp and 2 lp + 1 at src + 2 lp
// (dst + 2 lp); point p of a line is p * src_ps (p * dst_ps) further
struct PairGeom {
    int npairs;
    int src_ps;
    int dst_ps;
};

__device__ __forceinline__ float2 ld2(const float *p) { return *reinterpret_cast<const float2 *>(p); }
__device__ __forceinline__ void st2(float *p, float2 v) { *reinterpret_cast<float2 *>(p) = v; }

// x[k] = the pair at point p0 + k, periodic wrap or zero outside [0, L)
template <int W>
__device__ __forceinline__ void load_window2(float2 (&x)[W], const float *in, int ps, int p0, int L, int per)
{
    if (p0 >= 0 && p0 + W <= L) {
        const float *b = in + p0 * ps;
#pragma unroll
        for (int k = 0; k < W; ++k) x[k] = ld2(b + k * ps);
    } else if (per) {
#pragma unroll
        for (int k = 0; k < W; ++k) x[k] = ld2(in + wrap_near(p0 + k, L) * ps);
    } else {
#pragma unroll
        for (int k = 0; k < W; ++k) {
            const int p = p0 + k;
            x[k] = ((unsigned)p < (unsigned)L) ? ld2(in + p * ps) : make_float2(0.f, 0.f);
        }
    }
}

// one window value, periodic wrap or zero outside [0, L)
__device__ __forceinline__ float2 load_point2(const float *in, int ps, int p, int L, int per, bool interior)
{
    if (interior) return ld2(in + p * ps);
    if (per) return ld2(in + wrap_near(p, L) * ps);
    return ((unsigned)p < (unsigned)L) ? ld2(in + p * ps) : make_float2(0.f, 0.f);
}

// store the SEG output pairs q0 + t of a segment, those in [0, L) only
// (all of them when FULL)
template <int SEG, bool FULL>
__device__ __forceinline__ void store_seg2(float *dst, const PairGeom &g, int lp, int q0, int L,
                                           const float2 (&acc)[SEG])
{
    float *out = dst + 2 * lp;
#pragma unroll
    for (int t = 0; t < SEG; ++t) {
        const int q = q0 + t;
        if (FULL || (unsigned)q < (unsigned)L) st2(out + q * g.dst_ps, acc[t]);
    }
}

// ---------------------------------------------------------------- synthesis
// y(2i+o) = sum_{l=-4..4} ch(2l+o) s(i-l) + cg(2l+o) w(i-l) on two lines at
// once (src line [s | w], the wavelet half at point H); free lines grow to
// F = 2N + 14 points stored at q = f + 7 (pass_syn's geometry)
template <int SEG>
__device__ __forceinline__ void pass2_syn(const float *src, float *dst, const PairGeom g, int N, int H, int per)
{
    using P = PV<float>;
    static_assert(SEG % 2 == 0, "even segment");
    constexpr int W = SEG / 2 + 8;
    const int F = fine_len(N, per);
    const int off = per ? 0 : 7;
    const int fstart = per ? 0 : -8;
    const int nseg = (F + off - fstart + SEG - 1) / SEG;
    auto full = [&](int s) {
        const int q0 = fstart + s * SEG + off;
        return q0 >= 0 && q0 + SEG <= F;
    };
    for_items2(g.npairs, nseg, full, [&](int lp, int s, auto full_t) {
        constexpr bool FULL = decltype(full_t)::value;
        const float *in = src + 2 * lp;
        const int f0 = fstart + s * SEG;
        const int c0 = f0 / 2;
        float2 xs[W], xw[W], acc[SEG];
        load_window2<W>(xs, in, g.src_ps, c0 - 4, N, per);
        load_window2<W>(xw, in + H * g.src_ps, g.src_ps, c0 - 4, N, per);
#pragma unroll
        for (int t = 0; t < SEG; ++t) {
            const int o = t & 1;
            const int ic = t / 2 + 4;
            float2 a = P::zero();
#pragma unroll
            for (int l = -4; l <= 4; ++l) {
                const int m = 2 * l + o;
                if (m < -7 || m > 8) continue;
                if (big_tap(WVL_CH_AT(m + 7), kSynSeedTap)) a = P::fma(Filt<float>::ch_lo(m + 7), xs[ic - l], a);
                if (big_tap(WVL_CG_AT(m + 7), kSynSeedTap)) a = P::fma(Filt<float>::cg_lo(m + 7), xw[ic - l], a);
            }
#pragma unroll
            for (int l = -4; l <= 4; ++l) {
                const int m = 2 * l + o;
                if (m < -7 || m > 8) continue;
                a = P::fma(Filt<float>::ch(m + 7), xs[ic - l], a);
                a = P::fma(Filt<float>::cg(m + 7), xw[ic - l], a);
            }
            acc[t] = a;
        }
        store_seg2<SEG, FULL>(dst, g, lp, f0 + off, F, acc);
    });
}

// ---------------------------------------------------------------- analysis
// c(i) = sum_l ch(l) y(2i+l), d(i) = sum_l cg(l) y(2i+l); dst line [c | d],
// the d half at point H
template <int SEG>
__device__ __forceinline__ void pass2_ana(const float *src, float *dst, const PairGeom g, int N, int H, int per)
{
    using P = PV<float>;
    static_assert(SEG % 2 == 0, "even segment");
    constexpr int HS = SEG / 2;
    constexpr int W = SEG + 14;
    const int F = fine_len(N, per);
    const int nseg = (N + HS - 1) / HS;
    auto full = [&](int s) { return s * HS + HS <= N; };
    for_items2(g.npairs, nseg, full, [&](int lp, int s, auto full_t) {
        constexpr bool FULL = decltype(full_t)::value;
        const float *in = src + 2 * lp;
        const int i0 = s * HS;
        float2 x[W], ci[HS], di[HS];
        load_window2<W>(x, in, g.src_ps, 2 * i0 - (per ? 7 : 0), F, per);
#pragma unroll
        for (int t = 0; t < HS; ++t) {
            float2 c = P::zero(), d = P::zero();
#pragma unroll
            for (int l = 0; l < 16; ++l) {
                c = P::fma(Filt<float>::ch(l), x[2 * t + l], c);
                d = P::fma(Filt<float>::cg(l), x[2 * t + l], d);
            }
            ci[t] = c;
            di[t] = d;
        }
        store_seg2<HS, FULL>(dst, g, lp, i0, N, ci);
        store_seg2<HS, FULL>(dst + H * g.dst_ps, g, lp, i0, N, di);
    });
}

// ---------------------------------------------------------------- magic filter
// MODE 0: mf periodic, 1: mft periodic, 2: mf grow (F -> F+15), 3: mft shrink
template <int SEG, int MODE>
__device__ __forceinline__ void pass2_mf(const float *src, float *dst, const PairGeom g, int Lin, int Lout)
{
    using P = PV<float>;
    constexpr int W = SEG + 15;
    constexpr int shift = MODE == 0 ? -8 : MODE == 1 ? -7 : MODE == 2 ? -15 : 0;
    constexpr bool rev = (MODE == 1 || MODE == 3);
    constexpr int per = (MODE <= 1);
    const int nseg = (Lout + SEG - 1) / SEG;
    auto full = [&](int s) { return s * SEG + SEG <= Lout; };
    for_items2(g.npairs, nseg, full, [&](int lp, int s, auto full_t) {
        constexpr bool FULL = decltype(full_t)::value;
        const float *in = src + 2 * lp;
        const int q0 = s * SEG;
        float2 x[W], acc[SEG];
        load_window2<W>(x, in, g.src_ps, q0 + shift, Lin, per);
#pragma unroll
        for (int t = 0; t < SEG; ++t) {
            float2 a = P::zero();
            if constexpr (!rev) {
#pragma unroll
                for (int k = 0; k < 16; ++k)
                    if (big_tap(WVL_MF_AT(k), kMfSeedTap)) a = P::fma(Filt<float>::mf_lo(k), x[t + k], a);
            }
#pragma unroll
            for (int k = 0; k < 16; ++k) a = P::fma(Filt<float>::mf(rev ? 15 - k : k), x[t + k], a);
            acc[t] = a;
        }
        store_seg2<SEG, FULL>(dst, g, lp, q0, Lout, acc);
    });
}

// ---------------------------------------------------------------- kinetic
// dst(q) = (ACC ? dst(q) : cshift src(q)) + scale sum_{l=-14..14} a(|l|) src(q+l)
// and ekin += sum_q src(q) scale conv(q) in FP64, as pass_kin.  The 29 taps are accumulated while the window
// streams through (each loaded pair feeds every output of the segment it
// reaches), so only the accumulators stay in registers.  The rounding of the
// taps biases the energy by sum_q x(q) sum_l lo(|l|) x(q+l); over a whole
// line, periodic or zero-padded, that is lo(0) C(0) + 2 sum_{l>0} lo(l) C(l)
// with C(l) = sum_q x(q) x(q-l), which each segment accumulates for its own
// outputs q from the window, for the kKinLags largest taps.
template <int SEG, bool ACC, bool EN = true>
__device__ __forceinline__ void pass2_kin(const float *src, float *dst, const PairGeom g, int L, int per, double scale_d,
                                          float cshift, double *ekin)
{
    using P = PV<float>;
    constexpr int W = SEG + 28;
    constexpr int NLAG = kKinLags;
    const float scale = (float)scale_d;
    const int nseg = (L + SEG - 1) / SEG;
    // interior segments (window inside the line, all outputs in it) take
    // plain loads and no per-output tests; the others wrap or zero-pad
    auto interior = [&](int s) {
        const int p0 = s * SEG - 14;
        return p0 >= 0 && p0 + W <= L;
    };
    double e = 0.0;
    for_items2(g.npairs, nseg, interior, [&](int lp, int s, auto int_t) {
        constexpr bool INT = decltype(int_t)::value;
        const float *in = src + 2 * lp;
        const int q0 = s * SEG;
        const int p0 = q0 - 14;
        const int nout = INT ? SEG : min(SEG, L - q0);
        const float *b = in + p0 * g.src_ps;
        float2 conv[SEG], lag[NLAG];
        [[maybe_unused]] float2 hist[NLAG];
#pragma unroll
        for (int t = 0; t < SEG; ++t) conv[t] = P::zero();
#pragma unroll
        for (int l = 0; l < NLAG; ++l) lag[l] = P::zero();
#pragma unroll
        for (int k = 0; k < W; ++k) {
            const float2 x = INT ? ld2(b + k * g.src_ps) : load_point2(in, g.src_ps, p0 + k, L, per, false);
#pragma unroll
            for (int t = 0; t < SEG; ++t) {
                const int l = k - 14 - t;   // tap offset of this value for output t
                if (l >= -14 && l <= 14) conv[t] = P::fma(Filt<float>::kin(l < 0 ? -l : l), x, conv[t]);
            }
            if constexpr (EN) {
#pragma unroll
                for (int j = NLAG - 1; j > 0; --j) hist[j] = hist[j - 1];
                hist[0] = x;
                // outputs of this segment: window positions 14 .. 14 + nout - 1
                if (k >= 14 && k < 14 + SEG && (INT || k - 14 < nout)) {
#pragma unroll
                    for (int l = 0; l < NLAG; ++l) lag[l] = P::fmav(x, hist[l], lag[l]);
                }
            }
        }
        float2 es = P::zero();
#pragma unroll
        for (int t = 0; t < SEG; ++t) {
            if (INT || t < nout) {
                const int q = q0 + t;
                float *o = dst + 2 * lp + q * g.dst_ps;
                float2 base;
                if constexpr (ACC) {
                    base = ld2(o);
                } else {
                    base = P::mul(cshift, ld2(in + q * g.src_ps));
                }
                if constexpr (EN) es = P::fmav(ld2(in + q * g.src_ps), conv[t], es);
                st2(o, P::fma(scale, conv[t], base));
            }
        }
        if constexpr (EN) {
            double el = (double)Filt<float>::kin_lo(0) * ((double)lag[0].x + (double)lag[0].y);
#pragma unroll
            for (int l = 1; l < NLAG; ++l)
                el += 2.0 * (double)Filt<float>::kin_lo(l) * ((double)lag[l].x + (double)lag[l].y);
            e += ((double)es.x + (double)es.y + el) * scale_d;
        }
    });
    if (EN && ekin) *ekin += e;
}

}  // namespace wvlh
