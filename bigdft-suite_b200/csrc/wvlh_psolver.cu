// Periodic Poisson solver in the interpolating-scaling-function (ISF) basis:
// the Hartree potential of a density on the real-space (ISF) grid of a
// periodic box, as the reference's PSolver computes it for periodic boundary
// conditions (kernel: Periodic_Kernel and fourtrans_isf,
// psolver/src/Build_Kernel.f90:16-262; solve: G_PoissonSolver with
// P_multkernel_NO, psolver/src/PSolver_Base_new.f90:337-2640; normalisation
// scal = 1/(n1 n2 n3), createKernel.f90:299; energy 0.5 sum(rho V) h^3,
// PSolver_Main.f90:403):
//
//   V^(k) = rho^(k) * phi^_x(k1) phi^_y(k2) phi^_z(k3) / (pi g^2),
//   g = (k1/L1, k2/L2, k3/L3) in cycles per bohr, L = n h,
//   V^(0) = offset / h^3,   V = (1/N) inverse FFT,
//
// with phi^ the Fourier transform of the order-16 ISF sampled at the grid's
// frequencies: phi^(p) = prod_{j>=1} H(p / 2^j), H the two-scale symbol
// 1/2 + sum over odd m of c_m cos(m p), c_m the 16-point Deslauriers-Dubuc
// (Lagrange) interpolation weights at the midpoint.
//
// FFTs are cuFFT (D2Z / Z2D, plans cached per grid); the kernel multiply, with
// the folded frequencies and the three 1D ISF factors, and the deterministic
// energy reduction are this file's kernels.
//
// Free boundary conditions (Free_Kernel, Build_Kernel.f90:985-1175; the
// solve of the zero-padded density, the reference's GPU path
// psolver/src/cufft.cu:614-710 with geo = 0): the kernel is built once per grid
// on the host (the 89-Gaussian expansion of 1/r, gequad :1679-1873, each
// Gaussian's 1D ISF overlaps and their cosine transforms) and summed into the
// (N3/2+1, N2/2+1, N1/2+1) Fourier table on the device; each solve pads rho
// into a persistent zero buffer, transforms (the 2D (y, x) transforms only
// over the occupied half of the z-planes), multiplies by the table,
// transforms back and crops the first octant.
//
// The exchange-correlation part of the Kohn-Sham potential is the reference's
// default LDA (ixc = 1: the Goedecker-Teter-Hutter Pade fit of the
// Ceperley-Alder data, Phys. Rev. B 54, 1703 (1996); ABINIT's xcspol,
// libABINIT/src/abi_xc_lowlevel/abi_xcspol.F90:105-250), spin-unpolarised,
// evaluated point by point in the same pass that adds V_H, V_ext and V_xc
// (updatePotential, bigdft/src/modules/rhopotential.f90:29-125).
#include <cuda_runtime.h>
#include <cufft.h>

#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "../../include/wvlh.h"
#include "wvlh_common.cuh"
#include "wvlh_internal.h"
#include "wvlh_objects.h"

namespace wvlh {
void set_last_error(int code);

// 16-point interpolation weights at the midpoint of the odd offsets
// -15, -13, ..., 15 (the order-16 ISF filter): c_m = prod_{i != m} (0 - i) / (m - i)
static double isf_weight(int m)
{
    double r = 1.0;
    for (int i = -15; i <= 15; i += 2)
        if (i != m) r *= (0.0 - i) / (double)(m - i);
    return r;
}

// H(p) = 1/2 + sum_{m odd, 1..15} c_m cos(m p) (fourtrans, Build_Kernel.f90:252-262)
static double isf_symbol(double p)
{
    static const double c[8] = {isf_weight(1), isf_weight(3), isf_weight(5), isf_weight(7),
                                isf_weight(9), isf_weight(11), isf_weight(13), isf_weight(15)};
    double h = 0.0;
    for (int j = 7; j >= 0; --j) h += c[j] * std::cos(p * (2 * j + 1));
    return 0.5 + h;
}

// phi^ at the frequencies i 2 pi / (2 n), i = 0..n (fourtrans_isf,
// Build_Kernel.f90:202-248): odd i by the infinite product (stopped where the
// factor is 1 to 1e-16), even i from i/2 by one more factor (dyadic grid).
static void fourtrans_isf(int n, std::vector<double> &f)
{
    const double twopi = 6.28318530717958647688;
    f.assign(n + 1, 0.0);
    f[0] = 1.0;
    for (int i = 1; i <= n; ++i) {
        if (i % 2 == 0) continue;
        const double p = i * twopi / (2.0 * n);
        double v = 1.0, q = p;
        for (;;) {
            q *= 0.5;
            const double h = isf_symbol(q);
            if (std::fabs(h - 1.0) <= 1e-16) break;
            v *= h;
        }
        f[i] = v;
        int j = i;
        q = p;
        for (;;) {
            j *= 2;
            if (j > n) break;
            f[j] = isf_symbol(q) * f[j / 2];
            q *= 2.0;
        }
    }
}

// one thread per complex coefficient of the D2Z output (n3, n2, n1/2 + 1)
__global__ void k_ps_multiply(int n1, int n2, int n3, double L1, double L2, double L3,
                              const double *__restrict__ fx, const double *__restrict__ fy,
                              const double *__restrict__ fz, double scal, double zero,
                              cufftDoubleComplex *__restrict__ z)
{
    const int nh = n1 / 2 + 1;
    const long long tot = (long long)n3 * n2 * nh;
    const double pi = 3.14159265358979323846;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
         e += (long long)gridDim.x * blockDim.x) {
        const int k1 = (int)(e % nh);
        const long long r = e / nh;
        const int k2 = (int)(r % n2), k3 = (int)(r / n2);
        const int p2 = k2 <= n2 / 2 ? k2 : n2 - k2, p3 = k3 <= n3 / 2 ? k3 : n3 - k3;   // |frequency|
        cufftDoubleComplex v = z[e];
        if (k1 == 0 && k2 == 0 && k3 == 0) {
            v.x = zero;
            v.y = 0.0;
        } else {
            const double g1 = k1 / L1, g2 = p2 / L2, g3 = p3 / L3;
            const double g = g1 * g1 + g2 * g2 + g3 * g3;
            const double f = fx[k1] * fy[p2] * fz[p3] / (pi * g) * scal;
            v.x *= f;
            v.y *= f;
        }
        z[e] = v;
    }
}

// fixed-order sum of rho * V: per-block partials, then one block over them
__global__ void k_ps_dot(long long n, const double *__restrict__ a, const double *__restrict__ b,
                         double *__restrict__ part)
{
    __shared__ double red[32];
    double s = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        s = fma(a[i], b[i], s);
    const double t = block_sum(s, red);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

__global__ void k_ps_sum(int n, const double *__restrict__ part, double scale, double *__restrict__ out)
{
    __shared__ double red[32];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += part[i];
    const double t = block_sum(s, red);
    if (threadIdx.x == 0) *out = t * scale;
}

// Teter 1993 paramagnetic parameters (abi_xcspol.F90:105-112) and
// rs = (3 / (4 pi rho))^(1/3) = rsfac rho^(-1/3) (abi_drivexc.F90:134, 213-224)
struct Teter93 {
    static constexpr double a0 = 0.4581652932831429, a1 = 2.217058676663745, a2 = 0.7405551735357053,
                            a3 = 0.01968227878617998;
    static constexpr double b1 = 1.0, b2 = 4.504130959426697, b3 = 1.110667363742916, b4 = 0.02359291751427506;
    static constexpr double rsfac = 0.6203504908994000;
};

// eps_xc and v_xc = d(rho eps_xc)/d rho of the total density rho (xcspol,
// nspden = 1, order 1: :229-250); rs keeps the sign of rho as abi_invcb does
__device__ __forceinline__ void teter_lda(double rho, double &eps, double &v)
{
    using T = Teter93;
    const double rs = T::rsfac * copysign(rcbrt(fabs(rho)), rho);
    const double n1 = T::a0 + rs * (T::a1 + rs * (T::a2 + rs * T::a3));
    const double d1 = rs * (T::b1 + rs * (T::b2 + rs * (T::b3 + rs * T::b4)));
    const double d1m1 = 1.0 / d1;
    eps = -n1 * d1m1;
    const double dn1 = T::a1 + rs * (2.0 * T::a2 + rs * (3.0 * T::a3));
    const double dd1 = T::b1 + rs * (2.0 * T::b2 + rs * (3.0 * T::b3 + rs * (4.0 * T::b4)));
    const double deps = -(dn1 + eps * dd1) * d1m1;
    v = eps - (1.0 / 3.0) * rs * deps;
}

// V_xc of every point (written, or added when ACC), per-block partial sums of
// eps rho and v rho (xc_energy_new, orbitals/xc.f90:888-917) in part[2 b + 0/1]
template <bool ACC>
__global__ void k_xc_lda(long long n, const double *__restrict__ rho, double *__restrict__ vxc,
                         double *__restrict__ part)
{
    __shared__ double red[32];
    double se = 0.0, sv = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double r = rho[i];
        double e, v;
        teter_lda(r, e, v);
        se = fma(e, r, se);
        sv = fma(v, r, sv);
        vxc[i] = ACC ? vxc[i] + v : v;
    }
    const double te = block_sum(se, red);
    const double tv = block_sum(sv, red);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = te;
        part[2 * blockIdx.x + 1] = tv;
    }
}

// the Kohn-Sham potential from V_H (in pot): pot = (V_H + V_ext) + V_xc, the
// order of H_potential's sum with pot_ion then updatePotential's axpy of V_XC;
// per-block partials of rho V_H, eps rho, v rho in part[3 b + 0/1/2]
__global__ void k_ks_combine(long long n, const double *__restrict__ rho, const double *__restrict__ vext,
                             double *__restrict__ pot, double *__restrict__ part)
{
    __shared__ double red[32];
    double sh = 0.0, se = 0.0, sv = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double r = rho[i], vh = pot[i];
        double e, v;
        teter_lda(r, e, v);
        sh = fma(vh, r, sh);
        se = fma(e, r, se);
        sv = fma(v, r, sv);
        pot[i] = (vext ? vh + vext[i] : vh) + v;
    }
    const double th = block_sum(sh, red);
    const double te = block_sum(se, red);
    const double tv = block_sum(sv, red);
    if (threadIdx.x == 0) {
        part[3 * blockIdx.x] = th;
        part[3 * blockIdx.x + 1] = te;
        part[3 * blockIdx.x + 2] = tv;
    }
}

// out[k] = scale[k] * sum over blocks of part[K b + k], blocks in a fixed order
template <int K>
__global__ void k_ps_sum_k(int nblk, const double *__restrict__ part, double s0, double s1, double s2,
                           double *__restrict__ out)
{
    __shared__ double red[32];
    const double sc[3] = {s0, s1, s2};
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = 0.0;
        for (int i = threadIdx.x; i < nblk; i += blockDim.x) s += part[K * i + k];
        const double t = block_sum(s, red);
        if (threadIdx.x == 0) out[k] = t * sc[k];
    }
}

struct PsPlan {
    cufftHandle fwd = 0, inv = 0;
    DevBuf spec, fac, part;
    // free boundary conditions: padded sizes, Fourier table, padded input
    // (zero outside the density's octant) and padded output
    int nf[3] = {0, 0, 0};
    cufftHandle fz = 0;     // z transforms over all (y, kx) columns
    DevBuf ker, pad, work, zin;
};

// ---------------------------------------------------------------- free BC kernel

// the order-16 ISF on [-15, 17] at spacing 1/16 (513 samples), by the cascade
// of scaling_function (scaling_function.f90:12-110, back_trans_16 :1232-1266):
// a unit value at 0 refined by doubling, even points kept, odd points the
// midpoint interpolation with the weights ch(odd)
static void isf_samples(std::vector<double> &x, std::vector<double> &y)
{
    const int ni = 32, nd = 512, mh = 9;   // itype 16: support 32, filter half-length (m = 18) / 2
    y.assign(nd + 1, 0.0);
    y[ni / 2 - 1] = 1.0;
    std::vector<double> prev, out;
    for (int nt = 2 * ni;; nt *= 2) {
        const int half = nt / 2;
        prev.assign(y.begin(), y.begin() + half);
        out.assign(nt, 0.0);
        for (int i = 0; i < half; ++i) {
            out[2 * i] = prev[i];
            double v = 0.0;
            for (int j = -mh; j < mh; ++j) {
                const int m = 2 * j + 1;
                if (m < -15 || m > 15) continue;
                const int ind = ((i - j) % half + half) % half;
                v += isf_weight(m < 0 ? -m : m) * prev[ind];
            }
            out[2 * i + 1] = v;
        }
        std::copy(out.begin(), out.end(), y.begin());
        if (nt == nd) break;
    }
    x.resize(nd + 1);
    for (int i = 0; i <= nd; ++i) x[i] = (double)i * ni / nd - (0.5 * ni - 1.0);
}

// k(i), i = -nr..nr (index i + nr): the overlap of phi(x - i) with
// exp(-p h^2 x^2) (gauss_conv_scf, Build_Kernel.f90:1597-1651): a sharp
// Gaussian's exponent divided by 4^n_iter, the Riemann sum over the ISF
// samples, then n_iter two-scale steps (scf_recursion_16,
// scaling_function.f90:1324-1356)
static void gauss_conv_isf(double p, double h, int nr, const std::vector<double> &xs, const std::vector<double> &ys,
                           std::vector<double> &k, std::vector<double> &k1)
{
    const double dx = 32.0 / (double)(xs.size() - 1);
    const double p0_cell = 1.0 / (h * h);
    int n_iter = (int)std::floor((std::log(p) - std::log(p0_cell)) / std::log(4.0) + 0.5);
    double p0 = p;
    if (n_iter <= 0)
        n_iter = 0;
    else
        p0 = p / std::pow(4.0, n_iter);
    const double x_limit = std::sqrt(634.71369555645470 / p0) / h;
    k.assign(2 * nr + 1, 0.0);
    for (int i = 0; i <= nr; ++i) {
        double v = 0.0;
        for (size_t s = 0; s < xs.size(); ++s) {
            const double a = xs[s] - i;
            if (std::fabs(a) < x_limit) v += ys[s] * std::exp(-p0 * (a * a * h * h));
        }
        k[nr + i] = k[nr - i] = v * dx;
        if (std::fabs(v) < 1e-18) break;
    }
    double ch[37];   // ch(-18..18)
    for (int j = -18; j <= 18; ++j) ch[j + 18] = j == 0 ? 1.0 : ((j & 1) && j >= -15 && j <= 15 ? isf_weight(j < 0 ? -j : j) : 0.0);
    for (int it = 0; it < n_iter; ++it) {
        k1 = k;
        std::fill(k.begin(), k.end(), 0.0);
        for (int i = 0; i <= nr; ++i) {
            double tot = 0.0;
            for (int j = -18; j <= 18; ++j) {
                const int ind = 2 * i - j;
                if (ind >= -nr && ind <= nr) tot += ch[j + 18] * k1[nr + ind];
            }
            if (tot == 0.0) break;
            k[nr + i] = k[nr - i] = 0.5 * tot;
        }
    }
}

// the smallest even length >= m whose factors are 2, 3, 5, 7 (the padded
// convolution is exact for any length >= twice the box)
static int fft_length(int m)
{
    for (int n = m + (m & 1);; n += 2) {
        int r = n;
        for (int f : {2, 3, 5, 7})
            while (r % f == 0) r /= f;
        if (r == 1) return n;
    }
}

// one table row per Gaussian g and direction d: C_d(k) = f(0) + 2 sum_{j=1}^{J-1}
// f(j) cos(2 pi k j / N_d), k = 0..N_d/2, J = min(n_range, N_d/2) (gauconv_ffts,
// Build_Kernel.f90:1184-1340, without the centring sign (-1)^k, which only
// moves the convolution's origin); rows laid out [g][x | y | z], then the
// weights w_g / a
static void free_kernel_tables(const int n0[3], const double h[3], const int nf[3], std::vector<double> &tab)
{
    const int ng = 89;
    const double a1 = h[0] * n0[0], a2 = h[1] * n0[1], a3 = h[2] * n0[2];
    const double ar2 = a1 * a1 + a2 * a2 + a3 * a3;
    const double factor = 1.0 / std::sqrt(ar2), factor2 = 1.0 / ar2;
    const int nr = std::max(std::max(std::max(n0[0], n0[1]), n0[2]), 32);
    std::vector<double> xs, ys, k, k1;
    isf_samples(xs, ys);
    const int len[3] = {nf[0] / 2 + 1, nf[1] / 2 + 1, nf[2] / 2 + 1};
    const int row = len[0] + len[1] + len[2];
    tab.assign((size_t)ng * row + ng, 0.0);
    std::vector<double> cs[3];
    int J[3];
    for (int d = 0; d < 3; ++d) {
        J[d] = std::min(nr, nf[d] / 2);
        cs[d].resize((size_t)len[d] * J[d]);
        for (int q = 0; q < len[d]; ++q)
            for (int j = 0; j < J[d]; ++j)
                cs[d][(size_t)q * J[d] + j] = std::cos(6.28318530717958647688 * ((long long)q * j % nf[d]) / nf[d]);
    }
    for (int g = 0; g < ng; ++g) {
        const double pg = WVL_GQ_P[g] * factor2;
        double *out = tab.data() + (size_t)g * row;
        for (int d = 0, off = 0; d < 3; off += len[d], ++d) {
            gauss_conv_isf(pg, h[d], nr, xs, ys, k, k1);
            const double *f = k.data() + nr;
            for (int q = 0; q < len[d]; ++q) {
                const double *c = cs[d].data() + (size_t)q * J[d];
                double s = 0.0;
                for (int j = 1; j < J[d]; ++j) s += f[j] * c[j];
                out[off + q] = f[0] + 2.0 * s;
            }
        }
        tab[(size_t)ng * row + g] = WVL_GQ_W[g] * factor;
    }
}

// K(k3, k2, k1) = sum over the Gaussians, last to first, of
// Cx(k1) (Cz(k3) (Cy(k2) w)) (Free_Kernel's accumulation order, :1146-1166)
__global__ void k_free_kernel(int l1, int l2, int l3, int ng, const double *__restrict__ tab, double *__restrict__ ker)
{
    const long long tot = (long long)l3 * l2 * l1;
    const int row = l1 + l2 + l3;
    const double *w = tab + (size_t)ng * row;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
         e += (long long)gridDim.x * blockDim.x) {
        const int i1 = (int)(e % l1);
        const long long r = e / l1;
        const int i2 = (int)(r % l2), i3 = (int)(r / l2);
        double s = 0.0;
        for (int g = ng - 1; g >= 0; --g) {
            const double *t = tab + (size_t)g * row;
            s += t[i1] * (t[l1 + l2 + i3] * (t[l1 + i2] * w[g]));
        }
        ker[e] = s;
    }
}

// rho (n3, n2, n1) into the corner of the padded (N3, N2, N1) buffer
__global__ void k_free_pad(int n1, int n2, int n3, int N1, int N2, const double *__restrict__ rho, double *__restrict__ pad)
{
    const long long tot = (long long)n3 * n2 * n1;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
         e += (long long)gridDim.x * blockDim.x) {
        const int i1 = (int)(e % n1);
        const long long r = e / n1;
        const int i2 = (int)(r % n2), i3 = (int)(r / n2);
        pad[((long long)i3 * N2 + i2) * N1 + i1] = rho[e];
    }
}

// the D2Z spectrum (N3, N2, N1/2+1) times scal K(|k3|, |k2|, k1)
__global__ void k_free_multiply(int N1, int N2, int N3, const double *__restrict__ ker, double scal,
                                cufftDoubleComplex *__restrict__ z)
{
    const int nh = N1 / 2 + 1, l2 = N2 / 2 + 1;
    const long long tot = (long long)N3 * N2 * nh;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
         e += (long long)gridDim.x * blockDim.x) {
        const int k1 = (int)(e % nh);
        const long long r = e / nh;
        const int k2 = (int)(r % N2), k3 = (int)(r / N2);
        const int p2 = k2 <= N2 / 2 ? k2 : N2 - k2, p3 = k3 <= N3 / 2 ? k3 : N3 - k3;
        const double f = ker[((long long)p3 * l2 + p2) * nh + k1] * scal;
        cufftDoubleComplex v = z[e];
        v.x *= f;
        v.y *= f;
        z[e] = v;
    }
}

// pot = the first octant of the padded result; per-block partials of rho pot
__global__ void k_free_crop(int n1, int n2, int n3, int N1, int N2, const double *__restrict__ work,
                            const double *__restrict__ rho, double *__restrict__ pot, double *__restrict__ part)
{
    __shared__ double red[32];
    const long long tot = (long long)n3 * n2 * n1;
    double s = 0.0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
         e += (long long)gridDim.x * blockDim.x) {
        const int i1 = (int)(e % n1);
        const long long r = e / n1;
        const int i2 = (int)(r % n2), i3 = (int)(r / n2);
        const double v = work[((long long)i3 * N2 + i2) * N1 + i1];
        if (part) s = fma(rho[e], v, s);
        pot[e] = v;
    }
    if (part) {
        const double t = block_sum(s, red);
        if (threadIdx.x == 0) part[blockIdx.x] = t;
    }
}

}  // namespace wvlh

using namespace wvlh;

// plans and buffers per (context, device, grid), kept for the process: an SCF
// loop solves on the same grid at every iteration
static std::mutex g_ps_mutex;
static std::map<std::tuple<const void *, int, int, int, int>, PsPlan *> g_ps_plans;
// free boundary conditions: per (context, device, grid, spacings)
static std::map<std::tuple<const void *, int, int, int, int, double, double, double>, PsPlan *> g_ps_free;

static void free_plan(PsPlan *pl)
{
    if (pl->fwd) cufftDestroy(pl->fwd);
    if (pl->inv) cufftDestroy(pl->inv);
    if (pl->fz) cufftDestroy(pl->fz);
    for (DevBuf *b : {&pl->spec, &pl->fac, &pl->part, &pl->ker, &pl->pad, &pl->work, &pl->zin}) b->release();
    delete pl;
}

namespace wvlh {
// the plans and buffers of a context, at its destruction (its stream is idle)
void psolver_release(const wvlh_ctx *ctx)
{
    std::lock_guard<std::mutex> lock(g_ps_mutex);
    for (auto it = g_ps_plans.begin(); it != g_ps_plans.end();) {
        if (std::get<0>(it->first) != (const void *)ctx) {
            ++it;
            continue;
        }
        free_plan(it->second);
        it = g_ps_plans.erase(it);
    }
    for (auto it = g_ps_free.begin(); it != g_ps_free.end();) {
        if (std::get<0>(it->first) != (const void *)ctx) {
            ++it;
            continue;
        }
        free_plan(it->second);
        it = g_ps_free.erase(it);
    }
}
}  // namespace wvlh

static const int kPsBlocks = 1184;   // 8 per SM on 148 SMs

static bool ps_args_ok(const int n[3], const double h[3])
{
    for (int k = 0; k < 3; ++k)
        if (n[k] < 16 || n[k] % 2 || !(h[k] > 0.0)) return false;   // the ISF needs 16 points, the kernel even sizes
    return true;
}

// V_H of rho into pot (D2Z, kernel multiply, Z2D on the context's stream);
// returns the grid's plan (its part buffer holds kPsBlocks * 3 doubles)
static int ps_hartree(wvlh_ctx *ctx, const int n[3], const double h[3], const double *rho, double *pot,
                      double offset, PsPlan **out)
{
    if (cudaSetDevice(ctx->device) != cudaSuccess) return WVLH_ERR_CUDA;
    const int n1 = n[0], n2 = n[1], n3 = n[2];
    const long long nc = (long long)n3 * n2 * (n1 / 2 + 1);
    PsPlan *pl;
    {
        std::lock_guard<std::mutex> lock(g_ps_mutex);
        const auto key = std::make_tuple((const void *)ctx, ctx->device, n1, n2, n3);
        auto it = g_ps_plans.find(key);
        if (it == g_ps_plans.end()) {
            // cuFFT's last dimension is the fastest: (n3, n2, n1) for x-fastest arrays
            cufftHandle f = 0, b = 0;
            if (cufftPlan3d(&f, n3, n2, n1, CUFFT_D2Z) != CUFFT_SUCCESS) return WVLH_ERR_CUDA;
            if (cufftPlan3d(&b, n3, n2, n1, CUFFT_Z2D) != CUFFT_SUCCESS) {
                cufftDestroy(f);
                return WVLH_ERR_CUDA;
            }
            PsPlan *np = new PsPlan();
            np->fwd = f;
            np->inv = b;
            it = g_ps_plans.emplace(key, np).first;
        }
        pl = it->second;
    }
    int rc;
    if ((rc = pl->spec.ensure(sizeof(cufftDoubleComplex) * (size_t)nc)) ||
        (rc = pl->fac.ensure(sizeof(double) * (size_t)(n1 / 2 + n2 / 2 + n3 / 2 + 3))) ||
        (rc = pl->part.ensure(sizeof(double) * (size_t)(3 * kPsBlocks + 3))))
        return rc;
    std::vector<double> fx, fy, fz;
    fourtrans_isf(n1 / 2, fx);
    fourtrans_isf(n2 / 2, fy);
    fourtrans_isf(n3 / 2, fz);
    std::vector<double> fac(fx);
    fac.insert(fac.end(), fy.begin(), fy.end());
    fac.insert(fac.end(), fz.begin(), fz.end());
    cudaStream_t st = ctx->stream;
    double *d_fac = (double *)pl->fac.p;
    cufftDoubleComplex *z = (cufftDoubleComplex *)pl->spec.p;
    cudaError_t e = cudaMemcpyAsync(d_fac, fac.data(), sizeof(double) * fac.size(), cudaMemcpyHostToDevice, st);
    bool ok = e == cudaSuccess && cufftSetStream(pl->fwd, st) == CUFFT_SUCCESS &&
              cufftSetStream(pl->inv, st) == CUFFT_SUCCESS &&
              cufftExecD2Z(pl->fwd, (cufftDoubleReal *)rho, z) == CUFFT_SUCCESS;
    const double vol = h[0] * h[1] * h[2];
    const double scal = 1.0 / ((double)n1 * (double)n2 * (double)n3);
    if (ok) {
        k_ps_multiply<<<kPsBlocks, 256, 0, st>>>(n1, n2, n3, n1 * h[0], n2 * h[1], n3 * h[2], d_fac,
                                                 d_fac + fx.size(), d_fac + fx.size() + fy.size(), scal,
                                                 offset / vol * scal, z);
        ok = cudaGetLastError() == cudaSuccess;
    }
    if (ok) ok = cufftExecZ2D(pl->inv, z, (cufftDoubleReal *)pot) == CUFFT_SUCCESS;
    if (!ok) return WVLH_ERR_CUDA;
    *out = pl;
    return WVLH_OK;
}

static int ps_fail(int rc)
{
    set_last_error(rc);
    return rc;
}

extern "C" int wvlh_psolver_periodic(wvlh_ctx *ctx, const int n[3], const double h[3], const double *rho,
                                     double *pot, double offset, double *eh)
{
    // the energy needs rho after the potential is written: no aliasing then
    if (!ctx || !n || !h || !rho || !pot || (eh && pot == rho) || !ps_args_ok(n, h)) return ps_fail(WVLH_ERR_ARG);
    PsPlan *pl = nullptr;
    int rc = ps_hartree(ctx, n, h, rho, pot, offset, &pl);
    if (rc) return ps_fail(rc);
    if (eh) {
        const long long npt = (long long)n[0] * n[1] * n[2];
        double *part = (double *)pl->part.p;
        k_ps_dot<<<kPsBlocks, 256, 0, ctx->stream>>>(npt, rho, pot, part);
        k_ps_sum<<<1, 1024, 0, ctx->stream>>>(kPsBlocks, part, 0.5 * h[0] * h[1] * h[2], eh);
        if (cudaGetLastError() != cudaSuccess) return ps_fail(WVLH_ERR_CUDA);
    }
    return WVLH_OK;
}

extern "C" int wvlh_xc_lda(wvlh_ctx *ctx, int64_t npts, const double *rho, double *vxc, int accumulate, double dvol,
                           double *energies)
{
    // each point is read before its own V_xc is written: vxc may be rho
    if (!ctx || npts < 0 || (npts > 0 && (!rho || !vxc))) return ps_fail(WVLH_ERR_ARG);
    if (cudaSetDevice(ctx->device) != cudaSuccess) return ps_fail(WVLH_ERR_CUDA);
    if (npts == 0 && !energies) return WVLH_OK;
    // the partials live in the context's grid-independent entry, key (0, 0, 0)
    PsPlan *pl;
    {
        std::lock_guard<std::mutex> lock(g_ps_mutex);
        const auto key = std::make_tuple((const void *)ctx, ctx->device, 0, 0, 0);
        auto it = g_ps_plans.find(key);
        if (it == g_ps_plans.end()) it = g_ps_plans.emplace(key, new PsPlan()).first;
        pl = it->second;
    }
    int rc = pl->part.ensure(sizeof(double) * (size_t)(3 * kPsBlocks + 3));
    if (rc) return ps_fail(rc);
    double *part = (double *)pl->part.p;
    cudaStream_t st = ctx->stream;
    if (accumulate)
        k_xc_lda<true><<<kPsBlocks, 256, 0, st>>>(npts, rho, vxc, part);
    else
        k_xc_lda<false><<<kPsBlocks, 256, 0, st>>>(npts, rho, vxc, part);
    if (energies) k_ps_sum_k<2><<<1, 1024, 0, st>>>(kPsBlocks, part, dvol, dvol, 0.0, energies);
    if (cudaGetLastError() != cudaSuccess) return ps_fail(WVLH_ERR_CUDA);
    return WVLH_OK;
}

extern "C" int wvlh_ks_potential_periodic(wvlh_ctx *ctx, const int n[3], const double h[3], const double *rho,
                                          const double *vext, double *pot, double *energies)
{
    // the combine pass reads rho and V_ext after V_H is written to pot
    if (!ctx || !n || !h || !rho || !pot || pot == rho || (vext && vext == pot) || !ps_args_ok(n, h))
        return ps_fail(WVLH_ERR_ARG);
    PsPlan *pl = nullptr;
    int rc = ps_hartree(ctx, n, h, rho, pot, 0.0, &pl);
    if (rc) return ps_fail(rc);
    const long long npt = (long long)n[0] * n[1] * n[2];
    const double dvol = h[0] * h[1] * h[2];
    double *part = (double *)pl->part.p;
    k_ks_combine<<<kPsBlocks, 256, 0, ctx->stream>>>(npt, rho, vext, pot, part);
    if (energies) k_ps_sum_k<3><<<1, 1024, 0, ctx->stream>>>(kPsBlocks, part, 0.5 * dvol, dvol, dvol, energies);
    if (cudaGetLastError() != cudaSuccess) return ps_fail(WVLH_ERR_CUDA);
    return WVLH_OK;
}

// the free-BC plan of a grid: the Fourier table of the kernel, the padded
// buffers and three cuFFT plans that skip the all-zero half of the padded
// volume: a 2D (y, x) D2Z over the n3 occupied z-planes only, a 1D z transform
// of every (y, kx) column (z slowest, one stride), and on the way back the
// same z transform then a 2D Z2D of the n3 planes that are kept.  Buffers:
// pad (n3, N2, N1) real, zero outside the density's (n2, n1) corner; zin
// (N3, N2, N1/2+1) complex, planes z >= n3 zero; spec (same shape) and work
// (n3, N2, N1) real.  The zero parts are written once; no transform writes
// into them.
static int ps_free_plan(wvlh_ctx *ctx, const int n[3], const double h[3], PsPlan **out)
{
    std::lock_guard<std::mutex> lock(g_ps_mutex);
    const auto key = std::make_tuple((const void *)ctx, ctx->device, n[0], n[1], n[2], h[0], h[1], h[2]);
    auto it = g_ps_free.find(key);
    if (it != g_ps_free.end()) {
        *out = it->second;
        return WVLH_OK;
    }
    PsPlan *pl = new PsPlan();
    for (int d = 0; d < 3; ++d) pl->nf[d] = fft_length(2 * n[d]);
    const int N1 = pl->nf[0], N2 = pl->nf[1], N3 = pl->nf[2];
    const int l1 = N1 / 2 + 1, l2 = N2 / 2 + 1, l3 = N3 / 2 + 1;
    const size_t npad = (size_t)n[2] * N2 * N1, nspec = (size_t)N3 * N2 * l1;
    int rc = WVLH_OK;
    {
        int n2d[2] = {N2, N1}, rin[2] = {N2, N1}, cin[2] = {N2, l1}, nz[1] = {N3};
        if (cufftPlanMany(&pl->fwd, 2, n2d, rin, 1, N2 * N1, cin, 1, N2 * l1, CUFFT_D2Z, n[2]) != CUFFT_SUCCESS ||
            cufftPlanMany(&pl->inv, 2, n2d, cin, 1, N2 * l1, rin, 1, N2 * N1, CUFFT_Z2D, n[2]) != CUFFT_SUCCESS ||
            cufftPlanMany(&pl->fz, 1, nz, nz, N2 * l1, 1, nz, N2 * l1, 1, CUFFT_Z2Z, N2 * l1) != CUFFT_SUCCESS)
            rc = WVLH_ERR_CUDA;
    }
    std::vector<double> tab;
    if (!rc) {
        free_kernel_tables(n, h, pl->nf, tab);
        if ((rc = pl->ker.ensure(sizeof(double) * (size_t)l3 * l2 * l1)) ||
            (rc = pl->fac.ensure(sizeof(double) * tab.size())) ||
            (rc = pl->pad.ensure(sizeof(double) * npad)) || (rc = pl->work.ensure(sizeof(double) * npad)) ||
            (rc = pl->spec.ensure(sizeof(cufftDoubleComplex) * nspec)) ||
            (rc = pl->zin.ensure(sizeof(cufftDoubleComplex) * nspec)) ||
            (rc = pl->part.ensure(sizeof(double) * (size_t)(3 * kPsBlocks + 3))))
            ;
    }
    if (!rc) {
        // synchronous set-up on the context's stream (once per grid)
        cudaStream_t st = ctx->stream;
        bool ok = cudaMemcpyAsync(pl->fac.p, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice, st) ==
                      cudaSuccess &&
                  cudaMemsetAsync(pl->pad.p, 0, sizeof(double) * npad, st) == cudaSuccess &&
                  cudaMemsetAsync(pl->zin.p, 0, sizeof(cufftDoubleComplex) * nspec, st) == cudaSuccess;
        if (ok) {
            k_free_kernel<<<kPsBlocks, 256, 0, st>>>(l1, l2, l3, 89, (const double *)pl->fac.p, (double *)pl->ker.p);
            ok = cudaGetLastError() == cudaSuccess && cudaStreamSynchronize(st) == cudaSuccess;
        }
        if (!ok) rc = WVLH_ERR_CUDA;
    }
    if (rc) {
        free_plan(pl);
        return rc;
    }
    g_ps_free.emplace(key, pl);
    *out = pl;
    return WVLH_OK;
}

static bool ps_free_args_ok(const int n[3], const double h[3])
{
    for (int k = 0; k < 3; ++k)
        if (n[k] < 2 || n[k] > 4096 || !(h[k] > 0.0)) return false;
    return true;
}

// V_H of rho with free boundary conditions into pot; eh partials when part
static int ps_free_hartree(wvlh_ctx *ctx, const int n[3], const double h[3], const double *rho, double *pot,
                           bool energy, PsPlan **out)
{
    if (cudaSetDevice(ctx->device) != cudaSuccess) return WVLH_ERR_CUDA;
    PsPlan *pl = nullptr;
    int rc = ps_free_plan(ctx, n, h, &pl);
    if (rc) return rc;
    const int N1 = pl->nf[0], N2 = pl->nf[1], N3 = pl->nf[2];
    cudaStream_t st = ctx->stream;
    double *pad = (double *)pl->pad.p, *work = (double *)pl->work.p;
    cufftDoubleComplex *z = (cufftDoubleComplex *)pl->spec.p, *zin = (cufftDoubleComplex *)pl->zin.p;
    k_free_pad<<<kPsBlocks, 256, 0, st>>>(n[0], n[1], n[2], N1, N2, rho, pad);
    bool ok = cudaGetLastError() == cudaSuccess && cufftSetStream(pl->fwd, st) == CUFFT_SUCCESS &&
              cufftSetStream(pl->inv, st) == CUFFT_SUCCESS && cufftSetStream(pl->fz, st) == CUFFT_SUCCESS &&
              cufftExecD2Z(pl->fwd, pad, zin) == CUFFT_SUCCESS &&               // (y, x) of the n3 planes
              cufftExecZ2Z(pl->fz, zin, z, CUFFT_FORWARD) == CUFFT_SUCCESS;     // z of every column
    if (ok) {
        const double scal = h[0] * h[1] * h[2] / ((double)N1 * (double)N2 * (double)N3);
        k_free_multiply<<<kPsBlocks, 256, 0, st>>>(N1, N2, N3, (const double *)pl->ker.p, scal, z);
        ok = cudaGetLastError() == cudaSuccess && cufftExecZ2Z(pl->fz, z, z, CUFFT_INVERSE) == CUFFT_SUCCESS &&
             cufftExecZ2D(pl->inv, z, work) == CUFFT_SUCCESS;                   // the n3 planes kept
    }
    if (ok) {
        k_free_crop<<<kPsBlocks, 256, 0, st>>>(n[0], n[1], n[2], N1, N2, work, rho, pot,
                                               energy ? (double *)pl->part.p : nullptr);
        ok = cudaGetLastError() == cudaSuccess;
    }
    if (!ok) return WVLH_ERR_CUDA;
    *out = pl;
    return WVLH_OK;
}

extern "C" int wvlh_psolver_free(wvlh_ctx *ctx, const int n[3], const double h[3], const double *rho, double *pot,
                                 double *eh)
{
    // rho is copied into the padded buffer before pot is written: pot may be
    // rho, unless the energy (which reads rho after) is asked for
    if (!ctx || !n || !h || !rho || !pot || (eh && pot == rho) || !ps_free_args_ok(n, h))
        return ps_fail(WVLH_ERR_ARG);
    PsPlan *pl = nullptr;
    int rc = ps_free_hartree(ctx, n, h, rho, pot, eh != nullptr, &pl);
    if (rc) return ps_fail(rc);
    if (eh) {
        k_ps_sum<<<1, 1024, 0, ctx->stream>>>(kPsBlocks, (const double *)pl->part.p, 0.5 * h[0] * h[1] * h[2], eh);
        if (cudaGetLastError() != cudaSuccess) return ps_fail(WVLH_ERR_CUDA);
    }
    return WVLH_OK;
}

extern "C" int wvlh_ks_potential_free(wvlh_ctx *ctx, const int n[3], const double h[3], const double *rho,
                                      const double *vext, double *pot, double *energies)
{
    if (!ctx || !n || !h || !rho || !pot || pot == rho || (vext && vext == pot) || !ps_free_args_ok(n, h))
        return ps_fail(WVLH_ERR_ARG);
    PsPlan *pl = nullptr;
    int rc = ps_free_hartree(ctx, n, h, rho, pot, false, &pl);
    if (rc) return ps_fail(rc);
    const long long npt = (long long)n[0] * n[1] * n[2];
    const double dvol = h[0] * h[1] * h[2];
    double *part = (double *)pl->part.p;
    k_ks_combine<<<kPsBlocks, 256, 0, ctx->stream>>>(npt, rho, vext, pot, part);
    if (energies) k_ps_sum_k<3><<<1, 1024, 0, ctx->stream>>>(kPsBlocks, part, 0.5 * dvol, dvol, dvol, energies);
    if (cudaGetLastError() != cudaSuccess) return ps_fail(WVLH_ERR_CUDA);
    return WVLH_OK;
}

extern "C" int64_t wvlh_psolver_free_tables(const int n[3], const double h[3], int nf[3], double *tab, int64_t cap)
{
    if (!n || !h || !nf || !ps_free_args_ok(n, h)) return ps_fail(WVLH_ERR_ARG);
    for (int d = 0; d < 3; ++d) nf[d] = fft_length(2 * n[d]);
    const int64_t need = 89LL * (nf[0] / 2 + nf[1] / 2 + nf[2] / 2 + 3) + 89;
    if (!tab) return need;
    if (cap < need) return ps_fail(WVLH_ERR_ARG);
    std::vector<double> t;
    free_kernel_tables(n, h, nf, t);
    std::copy(t.begin(), t.end(), tab);
    return need;
}
