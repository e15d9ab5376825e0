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
#include <thread>
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

// the D2Z spectrum (N3, N2, N1/2+1) times scal K(|k3|, |k2|, k1), K a real
// table (N3/2+1, N2/2+1, N1/2+1) of the kernel; one warp per spectrum row.
// zero_term: the k = 0 coefficient is set to (zero, 0) instead (the periodic
// solver's offset term)
__global__ void k_table_multiply(int N1, int N2, int N3, const double *__restrict__ ker, double scal, int zero_term,
                                 double zero, cufftDoubleComplex *__restrict__ z)
{
    const int nh = N1 / 2 + 1, l2 = N2 / 2 + 1;
    const int lane = threadIdx.x & 31;
    const int nrow = N3 * N2;
    const int w0 = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), nw = (int)((gridDim.x * blockDim.x) >> 5);
    for (int r = w0; r < nrow; r += nw) {
        const int k3 = r / N2, k2 = r - k3 * N2;
        const int p2 = k2 <= N2 / 2 ? k2 : N2 - k2, p3 = k3 <= N3 / 2 ? k3 : N3 - k3;   // |frequency|
        const double *kr = ker + ((size_t)p3 * l2 + p2) * nh;
        cufftDoubleComplex *zr = z + (size_t)r * nh;
        for (int k1 = lane; k1 < nh; k1 += 32) {
            cufftDoubleComplex v = zr[k1];
            const double f = kr[k1] * scal;
            v.x *= f;
            v.y *= f;
            if (zero_term && r == 0 && k1 == 0) {
                v.x = zero;
                v.y = 0.0;
            }
            zr[k1] = v;
        }
    }
}

// Each block writes its K partial sums v[k] (block_sum over the threads) to
// part[K b + k]; the last block to arrive (counted in *cnt) sums the blocks'
// partials in block order and writes out[k] = sc[k] * sum, then resets the
// counter for the next launch.  The order of every sum is fixed by the grid:
// deterministic.  Called by every thread of the block.
template <int K>
__device__ __forceinline__ void finish_partials(const double (&v)[K], double *__restrict__ part, unsigned int *cnt,
                                                const double (&sc)[K], double *__restrict__ out, double *red)
{
    __shared__ bool last;
    double t[K];
#pragma unroll
    for (int k = 0; k < K; ++k) t[k] = block_sum(v[k], red);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) part[K * blockIdx.x + k] = t[k];
        __threadfence();
        last = atomicAdd(cnt, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = 0.0;
        for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) s += __ldcg(part + K * i + k);
        const double r = block_sum(s, red);
        if (threadIdx.x == 0) out[k] = r * sc[k];
    }
    if (threadIdx.x == 0) *cnt = 0u;
}

// out = scale sum(a b) (the Hartree energy of the periodic solver)
__global__ void k_ps_dot(long long n, const double *__restrict__ a, const double *__restrict__ b,
                         double *__restrict__ part, unsigned int *cnt, double scale, double *__restrict__ out)
{
    __shared__ double red[32];
    double s = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        s = fma(a[i], b[i], s);
    const double v[1] = {s}, sc[1] = {scale};
    finish_partials<1>(v, part, cnt, sc, out, red);
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

// V_xc of every point (written, or added when ACC); with out, out[0..1] =
// dvol (sum eps rho, sum v rho) (xc_energy_new, orbitals/xc.f90:888-917)
template <bool ACC>
__global__ void k_xc_lda(long long n, const double *__restrict__ rho, double *__restrict__ vxc,
                         double *__restrict__ part, unsigned int *cnt, double dvol, double *__restrict__ out)
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
    if (!out) return;
    const double v[2] = {se, sv}, sc[2] = {dvol, dvol};
    finish_partials<2>(v, part, cnt, sc, out, red);
}

// the Kohn-Sham potential from V_H (in pot): pot = (V_H + V_ext) + V_xc, the
// order of H_potential's sum with pot_ion then updatePotential's axpy of V_XC;
// with out, out[0..2] = (0.5 dvol sum rho V_H, dvol sum eps rho, dvol sum v rho)
__global__ void k_ks_combine(long long n, const double *__restrict__ rho, const double *__restrict__ vext,
                             double *__restrict__ pot, double *__restrict__ part, unsigned int *cnt, double dvol,
                             double *__restrict__ out, const double *__restrict__ rhocore = nullptr)
{
    __shared__ double red[32];
    double sh = 0.0, se = 0.0, sv = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double r = rho[i], vh = pot[i];
        // a core density joins the valence one for XC only (XC_potential adds it
        // before the functional and takes its share out of int rho V_xc)
        const double rx = rhocore ? r + rhocore[i] : r;
        double e, v;
        teter_lda(rx, e, v);
        sh = fma(vh, r, sh);
        se = fma(e, rx, se);
        sv = fma(v, r, sv);
        pot[i] = (vext ? vh + vext[i] : vh) + v;
    }
    if (!out) return;
    const double v[3] = {sh, se, sv}, sc[3] = {0.5 * dvol, dvol, dvol};
    finish_partials<3>(v, part, cnt, sc, out, red);
}

// ferromagnetic - paramagnetic differences of the fit (abi_xcspol.F90:113-116)
struct Teter93Spin {
    static constexpr double da0 = 0.119086804055547, da1 = 0.6157402568883345, da2 = 0.1574201515892867,
                            da3 = 0.003532336663397157;
    static constexpr double db1 = 0.0, db2 = 0.2673612973836267, db3 = 0.2052004607777787,
                            db4 = 0.004200005045691381;
    static constexpr double alpha = 1.0 - 1.0e-6;
};

// eps_xc and v_xc of both spins (xcspol, nspden = 2, order 1, :355-395):
// zeta = 2 up / rho - 1, the parameters interpolated with
// f(zeta) = ((1 + a z)^(4/3) + (1 - a z)^(4/3) - 2) / (2^(4/3) - 2),
// v_up/dn = v_para - (zeta -/+ 1) d eps / d zeta
__device__ __forceinline__ void teter_lsda(double up, double dn, double &eps, double &vu, double &vd)
{
    using T = Teter93;
    using S = Teter93Spin;
    const double rho = up + dn;
    const double zet = 2.0 * up / rho - 1.0;
    const double rs = T::rsfac * copysign(rcbrt(fabs(rho)), rho);
    const double fact = 1.0 / (2.5198420997897464 - 2.0);   // 2^(4/3) = 2.5198420997897464
    const double zp = 1.0 + zet * S::alpha, zm = 1.0 - zet * S::alpha;
    const double zp3 = cbrt(zp), zm3 = cbrt(zm);
    const double fxc = (zp * zp3 + zm * zm3 - 2.0) * fact;
    const double a0 = T::a0 + fxc * S::da0, a1 = T::a1 + fxc * S::da1, a2 = T::a2 + fxc * S::da2,
                 a3 = T::a3 + fxc * S::da3;
    const double b1 = T::b1 + fxc * S::db1, b2 = T::b2 + fxc * S::db2, b3 = T::b3 + fxc * S::db3,
                 b4 = T::b4 + fxc * S::db4;
    const double n1 = a0 + rs * (a1 + rs * (a2 + rs * a3));
    const double d1 = rs * (b1 + rs * (b2 + rs * (b3 + rs * b4)));
    const double d1m1 = 1.0 / d1;
    eps = -n1 * d1m1;
    const double dn1 = a1 + rs * (2.0 * a2 + rs * (3.0 * a3));
    const double dd1 = b1 + rs * (2.0 * b2 + rs * (3.0 * b3 + rs * (4.0 * b4)));
    const double vp = eps - (1.0 / 3.0) * rs * (-(dn1 + eps * dd1) * d1m1);
    const double dfdz = (4.0 / 3.0) * S::alpha * (zp3 - zm3) * fact;
    const double dn1df = S::da0 + rs * (S::da1 + rs * (S::da2 + rs * S::da3));
    const double dd1df = rs * (S::db1 + rs * (S::db2 + rs * (S::db3 + rs * S::db4)));
    const double dedz = dfdz * (-(dn1df + eps * dd1df) * d1m1);
    vu = vp - (zet - 1.0) * dedz;
    vd = vp - (zet + 1.0) * dedz;
}

// V_xc of both spins (written, or added when ACC); with out, out[0..1] =
// dvol (sum eps rho, sum_sigma v_sigma rho_sigma) (xc_energy_new :888-917)
template <bool ACC>
__global__ void k_xc_lsda(long long n, const double *__restrict__ up, const double *__restrict__ dn,
                          double *__restrict__ vu, double *__restrict__ vd, double *__restrict__ part,
                          unsigned int *cnt, double dvol, double *__restrict__ out)
{
    __shared__ double red[32];
    double se = 0.0, sv = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double ru = up[i], rd = dn[i];
        double e, a, b;
        teter_lsda(ru, rd, e, a, b);
        se = fma(e, ru + rd, se);
        sv = fma(a, ru, fma(b, rd, sv));
        vu[i] = ACC ? vu[i] + a : a;
        vd[i] = ACC ? vd[i] + b : b;
    }
    if (!out) return;
    const double v[2] = {se, sv}, sc[2] = {dvol, dvol};
    finish_partials<2>(v, part, cnt, sc, out, red);
}

// the total density of the two spins (the Hartree solve's input)
__global__ void k_spin_total(long long n, const double *__restrict__ up, const double *__restrict__ dn,
                             double *__restrict__ tot)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        tot[i] = up[i] + dn[i];
}

// the spin-polarised Kohn-Sham potentials from V_H (in pu): p_sigma =
// (V_H + V_ext) + V_xc,sigma (updatePotential with nspin = 2); with out,
// out[0..2] = (0.5 dvol sum rho V_H, dvol sum eps rho, dvol sum_sigma v rho)
__global__ void k_ks_combine_spin(long long n, const double *__restrict__ up, const double *__restrict__ dn,
                                  const double *__restrict__ vext, double *__restrict__ pu, double *__restrict__ pd,
                                  double *__restrict__ part, unsigned int *cnt, double dvol, double *__restrict__ out,
                                  const double *__restrict__ rhocore = nullptr)
{
    __shared__ double red[32];
    double sh = 0.0, se = 0.0, sv = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double ru = up[i], rd = dn[i], vh = pu[i];
        const double hc = rhocore ? 0.5 * rhocore[i] : 0.0;   // half the core density on each spin
        double e, a, b;
        teter_lsda(ru + hc, rd + hc, e, a, b);
        const double r = ru + rd;
        sh = fma(vh, r, sh);
        se = fma(e, (ru + hc) + (rd + hc), se);
        sv = fma(a, ru, fma(b, rd, sv));
        const double base = vext ? vh + vext[i] : vh;
        pu[i] = base + a;
        pd[i] = base + b;
    }
    if (!out) return;
    const double v[3] = {sh, se, sv}, sc[3] = {0.5 * dvol, dvol, dvol};
    finish_partials<3>(v, part, cnt, sc, out, red);
}

struct PsPlan {
    cufftHandle fwd = 0, inv = 0;
    DevBuf spec, fac, part, cnt;          // cnt: the block-arrival counter of the energy sums
    bool cnt_zeroed = false;
    double tab_h[3] = {0.0, 0.0, 0.0};   // spacings the periodic kernel table in ker was built for
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

// pot = the first octant of the padded result (rows (i3, i2) of the
// (n3, N2, N1) output); with out, *out = scale sum(rho pot)
__global__ void k_free_crop(int n1, int n2, int n3, int N1, int N2, const double *__restrict__ work,
                            const double *__restrict__ rho, double *__restrict__ pot, double *__restrict__ part,
                            unsigned int *cnt, double scale, double *__restrict__ out)
{
    __shared__ double red[32];
    const int lane = threadIdx.x & 31;
    const int nrow = n3 * n2;
    const int w0 = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), nw = (int)((gridDim.x * blockDim.x) >> 5);
    double s = 0.0;
    for (int r = w0; r < nrow; r += nw) {
        const int i3 = r / n2, i2 = r - i3 * n2;
        const double *wr = work + ((size_t)i3 * N2 + i2) * N1;
        const size_t o = (size_t)r * n1;
        for (int i1 = lane; i1 < n1; i1 += 32) {
            const double v = wr[i1];
            if (out) s = fma(rho[o + i1], v, s);
            pot[o + i1] = v;
        }
    }
    if (!out) return;
    const double v[1] = {s}, sc[1] = {scale};
    finish_partials<1>(v, part, cnt, sc, out, red);
}


// ---------------------------------------------------------------- surface BC kernel
// (x and z periodic, y free: Surfaces_Kernel, Build_Kernel.f90:279-731)

// closed 9-point Newton-Cotes weights, the order-8 composite rule of
// calculates_green_opt (intorder 8, cpol(:, 8) times 8)
static const double kNC9[9] = {989.0 * 4.0 / 14175.0,  5888.0 * 4.0 / 14175.0, -928.0 * 4.0 / 14175.0,
                               10496.0 * 4.0 / 14175.0, -4540.0 * 4.0 / 14175.0, 10496.0 * 4.0 / 14175.0,
                               -928.0 * 4.0 / 14175.0,  5888.0 * 4.0 / 14175.0, 989.0 * 4.0 / 14175.0};

// the ISF at spacing 32 / nd on [-15, 17] (the cascade of isf_samples, to nd points)
static void isf_samples_n(int nd, std::vector<double> &x, std::vector<double> &y)
{
    const int ni = 32, mh = 9;
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
                v += isf_weight(m < 0 ? -m : m) * prev[((i - j) % half + half) % half];
            }
            out[2 * i + 1] = v;
        }
        std::copy(out.begin(), out.end(), y.begin());
        if (nt == nd) break;
    }
    x.resize(nd + 1);
    for (int i = 0; i <= nd; ++i) x[i] = (double)i * ni / nd - (0.5 * ni - 1.0);
}

// n_iter two-scale steps k(i) <- 1/2 sum_j ch(j) k(2i - j) on k(-nr..nr),
// stopping at the first zero sum (scf_recursion_16)
static void two_scale_steps(std::vector<double> &k, int nr, int n_iter, std::vector<double> &k1)
{
    double ch[37];
    for (int j = -18; j <= 18; ++j)
        ch[j + 18] = j == 0 ? 1.0 : ((j & 1) && j >= -15 && j <= 15 ? isf_weight(j < 0 ? -j : j) : 0.0);
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

struct IsfFine {
    std::vector<double> x, y;
    int n_scf = 0, izero = 0;
    double hres = 0.0;
    IsfFine()
    {
        isf_samples_n(2048, x, y);
        n_scf = 2048;
        hres = 32.0 / n_scf;
        while (izero < n_scf && x[izero] < 0.0) ++izero;
    }
    // the right-half integral from x = 0 of y g (panels while 9 points and one
    // more remain, then the leftover points with the first weights)
    template <class G> double right(G g) const
    {
        double s = 0.0;
        int iv = izero;
        for (; iv < n_scf - 9; iv += 8)
            for (int i = 0; i < 9; ++i) s += kNC9[i] * y[iv + i] * g(x[iv + i]);
        for (int i = 0; iv + i < n_scf; ++i) s += kNC9[i] * y[iv + i] * g(x[iv + i]);
        return s;
    }
    // the integral of y g over the unit segment [j-1, j] (j >= 1), 0 past the samples
    template <class G> double segment(int j, G g) const
    {
        const int s0 = izero + 64 * (j - 1);
        if (s0 >= n_scf) return 0.0;
        double s = 0.0;
        for (int p = 0; p < 8; ++p)
            for (int i = 0; i < 9; ++i) s += kNC9[i] * y[s0 + 8 * p + i] * g(x[s0 + 8 * p + i]);
        return s;
    }
};

// g(j) = integral of phi(x - j) exp(-mu |x|), j = 0..n-1 (calculates_green_opt,
// Build_Kernel.f90:734-864)
static void green_surface(int n, double mu, const IsfFine &f, std::vector<double> &out, std::vector<double> &g,
                          std::vector<double> &tmp)
{
    int n_iter = 0;
    double mu0 = mu;
    if (mu > 0.2) {
        n_iter = 1;
        while (mu / std::pow(2.0, n_iter) > 0.2) ++n_iter;
        mu0 = mu / std::pow(2.0, n_iter);
    }
    int nrec = (1 << n_iter) * n;
    g.assign(2 * nrec + 1, 0.0);
    double gright = f.hres * f.right([mu0](double x) { return std::exp(-mu0 * x); });
    double gleft = gright;
    g[nrec] = gleft + gright;
    const int nseg = (f.n_scf - f.izero) / 64;   // unit segments holding samples
    const double em = std::exp(-mu0), ep = std::exp(mu0);
    int nr = nrec;
    for (int ik = 1; ik <= nrec; ++ik) {
        const double lt = f.segment(ik, [mu0](double x) { return std::exp(mu0 * x); });
        const double rt = f.segment(ik, [mu0](double x) { return std::exp(-mu0 * x); });
        gleft = em * (gleft + f.hres * std::exp(-mu0 * (ik - 1)) * lt);
        gright = ik < nseg ? ep * (gright - f.hres * std::exp(mu0 * (ik - 1)) * rt) : 0.0;
        g[nrec + ik] = g[nrec - ik] = gleft + gright;
        if (std::fabs(gleft + gright) <= 1e-20) {
            nr = ik;
            break;
        }
    }
    std::vector<double> k(g.begin() + (nrec - nr), g.begin() + (nrec + nr + 1));
    two_scale_steps(k, nr, n_iter, tmp);
    out.assign(n, 0.0);
    for (int j = 0; j < std::min(n, nr); ++j) out[j] = k[nr + j];
}

// g(j) = integral of phi(x) |x - j|, j = 0..n-1 (calculates_green_opt_muzero,
// Build_Kernel.f90:867-953)
static void green_surface_mu0(int n, const IsfFine &f, std::vector<double> &out)
{
    double gr1 = f.hres * f.right([](double x) { return x; });
    double gl1 = -gr1, gl0 = 0.5, gr0 = 0.5;
    out.assign(n, 0.0);
    out[0] = 2.0 * gr1;
    for (int ik = 1; ik < n; ++ik) {
        const double c0 = f.hres * f.segment(ik, [](double) { return 1.0; });
        const double c1 = f.hres * f.segment(ik, [](double x) { return x; });
        gl0 += c0;
        gl1 += c1;
        gr0 -= c0;
        gr1 -= c1;
        out[ik] = ik * (gl0 - gr0) + gr1 - gl1;
    }
}

// the (n3/2+1, N2/2+1, n1/2+1) table K(k3, ky, k1): for each in-plane
// frequency mu = 2 pi h_y |g|, the Green's function along y (-h_y/(2 mu) g,
// or h_y/2 g at mu = 0) on the n2 points, cosine-transformed on N2 (without the
// reference's centring sign (-1)^k); rows of k3 computed on the host's threads
static void surface_kernel_table(const int n[3], const double h[3], int N2, std::vector<double> &tab)
{
    static const IsfFine f;
    const int n1 = n[0], n2 = n[1], n3 = n[2];
    const int nr = std::max(n2, 32), l1 = n1 / 2 + 1, l2 = N2 / 2 + 1, l3 = n3 / 2 + 1, J = std::min(n2, N2 / 2);
    std::vector<double> cs((size_t)l2 * J);
    for (int q = 0; q < l2; ++q)
        for (int j = 0; j < J; ++j)
            cs[(size_t)q * J + j] = std::cos(6.28318530717958647688 * ((long long)q * j % N2) / N2);
    tab.assign((size_t)l3 * l2 * l1, 0.0);
    auto rows = [&](int r0, int r1) {
        std::vector<double> v, g, tmp;
        for (int k3 = r0; k3 < r1; ++k3)
            for (int k1 = 0; k1 < l1; ++k1) {
                const double g1 = k1 / (n1 * h[0]), g3 = k3 / (n3 * h[2]);
                const double mu = h[1] * 6.28318530717958647688 * std::sqrt(g1 * g1 + g3 * g3);
                double sc;
                if (k1 == 0 && k3 == 0) {
                    green_surface_mu0(nr, f, v);
                    sc = 0.5 * h[1];
                } else {
                    green_surface(nr, mu, f, v, g, tmp);
                    sc = -0.5 * h[1] / mu;
                }
                for (int q = 0; q < l2; ++q) {
                    const double *c = cs.data() + (size_t)q * J;
                    double s = 0.0;
                    for (int j = 1; j < J; ++j) s += sc * v[j] * c[j];
                    tab[((size_t)k3 * l2 + q) * l1 + k1] = sc * v[0] + 2.0 * s;
                }
            }
    };
    const int nt = std::max(1, std::min(l3, (int)std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t) th.emplace_back(rows, (int)((long long)l3 * t / nt), (int)((long long)l3 * (t + 1) / nt));
    for (auto &x : th) x.join();
}


// ---------------------------------------------------------------- wire BC kernel
// (z periodic, x and y free: Wires_Kernel, Build_Kernel.f90:2244-2364)

// K(kz, ky, kx), (n_z/2+1, Ny/2+1, Nx/2+1): per z frequency the plane's Green's
// function as 144 separable Gaussians (log(mu0 r) at k_z = 0 with -log(mu0)
// added at k = 0, -K0(mu r) otherwise), each through the ISF overlaps and
// cosine transforms of the free kernel on the padded lengths; summed in the
// reference's order (Gaussian 1 to 144, (w C_x) C_y); k_z rows on the host's threads
static void wire_kernel_table(const int n[3], const double h[3], int Nx, int Ny, std::vector<double> &tab)
{
    const int nx = n[0], ny = n[1], nz = n[2];
    const int nr = std::max(std::max(nx, ny), 32);
    const int lx = Nx / 2 + 1, ly = Ny / 2 + 1, lz = nz / 2 + 1;
    const int Jx = std::min(nr, Nx / 2), Jy = std::min(nr, Ny / 2);
    std::vector<double> xs, ys;
    isf_samples(xs, ys);
    std::vector<double> csx((size_t)lx * Jx), csy((size_t)ly * Jy);
    for (int q = 0; q < lx; ++q)
        for (int j = 0; j < Jx; ++j) csx[(size_t)q * Jx + j] = std::cos(6.28318530717958647688 * ((long long)q * j % Nx) / Nx);
    for (int q = 0; q < ly; ++q)
        for (int j = 0; j < Jy; ++j) csy[(size_t)q * Jy + j] = std::cos(6.28318530717958647688 * ((long long)q * j % Ny) / Ny);
    tab.assign((size_t)lz * ly * lx, 0.0);
    auto rows = [&](int r0, int r1) {
        std::vector<double> k, k1, cx(lx), cy(ly);
        for (int kz = r0; kz < r1; ++kz) {
            double mu;
            const double *alpha, *wt;
            double wsign;
            if (kz == 0) {
                mu = 1.0 / std::sqrt((h[0] * (nx + 32)) * (h[0] * (nx + 32)) + (h[1] * (ny + 32)) * (h[1] * (ny + 32)));
                alpha = WVL_WIRE_P1;
                wt = WVL_WIRE_W1;
                wsign = 1.0;
            } else {
                mu = 6.28318530717958647688 / nz * kz / h[2];
                alpha = WVL_WIRE_P2;
                wt = WVL_WIRE_W2;
                wsign = -1.0;   // -K0
            }
            double *out = tab.data() + (size_t)kz * ly * lx;
            for (int g = 0; g < 144; ++g) {
                const double p = alpha[g] * mu * mu;
                gauss_conv_isf(p, h[0], nr, xs, ys, k, k1);
                for (int q = 0; q < lx; ++q) {
                    const double *c = csx.data() + (size_t)q * Jx;
                    double s = 0.0;
                    for (int j = 1; j < Jx; ++j) s += k[nr + j] * c[j];
                    cx[q] = k[nr] + 2.0 * s;
                }
                gauss_conv_isf(p, h[1], nr, xs, ys, k, k1);
                for (int q = 0; q < ly; ++q) {
                    const double *c = csy.data() + (size_t)q * Jy;
                    double s = 0.0;
                    for (int j = 1; j < Jy; ++j) s += k[nr + j] * c[j];
                    cy[q] = k[nr] + 2.0 * s;
                }
                const double w = wsign * wt[g];
                for (int qy = 0; qy < ly; ++qy)
                    for (int qx = 0; qx < lx; ++qx) out[(size_t)qy * lx + qx] += (w * cx[qx]) * cy[qy];
            }
            if (kz == 0) out[0] -= (double)Nx * (double)Ny * std::log(mu);
        }
    };
    const int nt = std::max(1, std::min(lz, (int)std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t) th.emplace_back(rows, (int)((long long)lz * t / nt), (int)((long long)lz * (t + 1) / nt));
    for (auto &x : th) x.join();
}

}  // namespace wvlh

using namespace wvlh;

// plans and buffers per (context, device, grid), kept for the process: an SCF
// loop solves on the same grid at every iteration
static std::mutex g_ps_mutex;
static std::map<std::tuple<const void *, int, int, int, int>, PsPlan *> g_ps_plans;
// free boundary conditions: per (context, device, grid, spacings)
static std::map<std::tuple<const void *, int, int, int, int, double, double, double>, PsPlan *> g_ps_free;
// surface and wire boundary conditions: the same key
static std::map<std::tuple<const void *, int, int, int, int, double, double, double>, PsPlan *> g_ps_surf;
static std::map<std::tuple<const void *, int, int, int, int, double, double, double>, PsPlan *> g_ps_wire;

static void free_plan(PsPlan *pl)
{
    if (pl->fwd) cufftDestroy(pl->fwd);
    if (pl->inv) cufftDestroy(pl->inv);
    if (pl->fz) cufftDestroy(pl->fz);
    for (DevBuf *b : {&pl->spec, &pl->fac, &pl->part, &pl->cnt, &pl->ker, &pl->pad, &pl->work, &pl->zin})
        b->release();
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
    for (auto *m : {&g_ps_free, &g_ps_surf, &g_ps_wire})
        for (auto it = m->begin(); it != m->end();) {
            if (std::get<0>(it->first) != (const void *)ctx) {
                ++it;
                continue;
            }
            free_plan(it->second);
            it = m->erase(it);
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

// the energy partials (3 per block) and the zeroed block-arrival counter
static int ps_energy_buffers(wvlh_ctx *ctx, PsPlan *pl)
{
    int rc;
    if ((rc = pl->part.ensure(sizeof(double) * (size_t)(3 * kPsBlocks + 3))) || (rc = pl->cnt.ensure(256)))
        return rc;
    if (!pl->cnt_zeroed) {
        if (cudaMemsetAsync(pl->cnt.p, 0, 256, ctx->stream) != cudaSuccess) return WVLH_ERR_CUDA;
        pl->cnt_zeroed = true;
    }
    return WVLH_OK;
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
    const int l1 = n1 / 2 + 1, l2 = n2 / 2 + 1, l3 = n3 / 2 + 1;
    if ((rc = pl->spec.ensure(sizeof(cufftDoubleComplex) * (size_t)nc)) ||
        (rc = pl->ker.ensure(sizeof(double) * (size_t)l3 * l2 * l1)) || (rc = ps_energy_buffers(ctx, pl)))
        return rc;
    cudaStream_t st = ctx->stream;
    if (pl->tab_h[0] != h[0] || pl->tab_h[1] != h[1] || pl->tab_h[2] != h[2]) {
        // the kernel table of this grid and spacing, (l3, l2, l1), k = 0 unused:
        // K = phi^_x phi^_y phi^_z / (pi g^2) at the folded frequencies
        std::vector<double> fx, fy, fz;
        fourtrans_isf(n1 / 2, fx);
        fourtrans_isf(n2 / 2, fy);
        fourtrans_isf(n3 / 2, fz);
        const double pi = 3.14159265358979323846, L1 = n1 * h[0], L2 = n2 * h[1], L3 = n3 * h[2];
        std::vector<double> tab((size_t)l3 * l2 * l1, 0.0);
        for (int p3 = 0; p3 < l3; ++p3)
            for (int p2 = 0; p2 < l2; ++p2)
                for (int k1 = 0; k1 < l1; ++k1) {
                    if (!k1 && !p2 && !p3) continue;
                    const double g1 = k1 / L1, g2 = p2 / L2, g3 = p3 / L3;
                    const double g = g1 * g1 + g2 * g2 + g3 * g3;
                    tab[((size_t)p3 * l2 + p2) * l1 + k1] = fx[k1] * fy[p2] * fz[p3] / (pi * g);
                }
        if (cudaMemcpyAsync(pl->ker.p, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice, st) !=
                cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return WVLH_ERR_CUDA;
        for (int d = 0; d < 3; ++d) pl->tab_h[d] = h[d];
    }
    cufftDoubleComplex *z = (cufftDoubleComplex *)pl->spec.p;
    bool ok = cufftSetStream(pl->fwd, st) == CUFFT_SUCCESS && cufftSetStream(pl->inv, st) == CUFFT_SUCCESS &&
              cufftExecD2Z(pl->fwd, (cufftDoubleReal *)rho, z) == CUFFT_SUCCESS;
    const double vol = h[0] * h[1] * h[2];
    const double scal = 1.0 / ((double)n1 * (double)n2 * (double)n3);
    if (ok) {
        k_table_multiply<<<kPsBlocks, 256, 0, st>>>(n1, n2, n3, (const double *)pl->ker.p, scal, 1,
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
        k_ps_dot<<<kPsBlocks, 256, 0, ctx->stream>>>(npt, rho, pot, (double *)pl->part.p, (unsigned int *)pl->cnt.p,
                                                     0.5 * h[0] * h[1] * h[2], eh);
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
    int rc = ps_energy_buffers(ctx, pl);
    if (rc) return ps_fail(rc);
    double *part = (double *)pl->part.p;
    unsigned int *cnt = (unsigned int *)pl->cnt.p;
    cudaStream_t st = ctx->stream;
    if (accumulate)
        k_xc_lda<true><<<kPsBlocks, 256, 0, st>>>(npts, rho, vxc, part, cnt, dvol, energies);
    else
        k_xc_lda<false><<<kPsBlocks, 256, 0, st>>>(npts, rho, vxc, part, cnt, dvol, energies);
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
    k_ks_combine<<<kPsBlocks, 256, 0, ctx->stream>>>(npt, rho, vext, pot, (double *)pl->part.p,
                                                     (unsigned int *)pl->cnt.p, dvol, energies);
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
            (rc = pl->zin.ensure(sizeof(cufftDoubleComplex) * nspec)) || (rc = ps_energy_buffers(ctx, pl)))
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

// V_H of rho with free boundary conditions into pot; with eh, *eh = the
// Hartree energy (reduced by the crop)
static int ps_free_hartree(wvlh_ctx *ctx, const int n[3], const double h[3], const double *rho, double *pot,
                           double *eh, PsPlan **out)
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
        k_table_multiply<<<kPsBlocks, 256, 0, st>>>(N1, N2, N3, (const double *)pl->ker.p, scal, 0, 0.0, z);
        ok = cudaGetLastError() == cudaSuccess && cufftExecZ2Z(pl->fz, z, z, CUFFT_INVERSE) == CUFFT_SUCCESS &&
             cufftExecZ2D(pl->inv, z, work) == CUFFT_SUCCESS;                   // the n3 planes kept
    }
    if (ok) {
        k_free_crop<<<kPsBlocks, 256, 0, st>>>(n[0], n[1], n[2], N1, N2, work, rho, pot, (double *)pl->part.p,
                                               (unsigned int *)pl->cnt.p, 0.5 * h[0] * h[1] * h[2], eh);
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
    int rc = ps_free_hartree(ctx, n, h, rho, pot, eh, &pl);
    if (rc) return ps_fail(rc);
    return WVLH_OK;
}

extern "C" int wvlh_ks_potential_free(wvlh_ctx *ctx, const int n[3], const double h[3], const double *rho,
                                      const double *vext, double *pot, double *energies)
{
    if (!ctx || !n || !h || !rho || !pot || pot == rho || (vext && vext == pot) || !ps_free_args_ok(n, h))
        return ps_fail(WVLH_ERR_ARG);
    PsPlan *pl = nullptr;
    int rc = ps_free_hartree(ctx, n, h, rho, pot, nullptr, &pl);
    if (rc) return ps_fail(rc);
    const long long npt = (long long)n[0] * n[1] * n[2];
    const double dvol = h[0] * h[1] * h[2];
    k_ks_combine<<<kPsBlocks, 256, 0, ctx->stream>>>(npt, rho, vext, pot, (double *)pl->part.p,
                                                     (unsigned int *)pl->cnt.p, dvol, energies);
    if (cudaGetLastError() != cudaSuccess) return ps_fail(WVLH_ERR_CUDA);
    return WVLH_OK;
}

extern "C" int64_t wvlh_psolver_free_tables(const int n[3], const double h[3], int nf[3], double *tab, int64_t cap)
{
    if (!n || !h || !nf || !ps_free_args_ok(n, h)) return -(int64_t)ps_fail(WVLH_ERR_ARG);
    for (int d = 0; d < 3; ++d) nf[d] = fft_length(2 * n[d]);
    const int64_t need = 89LL * (nf[0] / 2 + nf[1] / 2 + nf[2] / 2 + 3) + 89;
    if (!tab) return need;
    if (cap < need) return -(int64_t)ps_fail(WVLH_ERR_ARG);
    std::vector<double> t;
    free_kernel_tables(n, h, nf, t);
    std::copy(t.begin(), t.end(), tab);
    return need;
}

extern "C" int wvlh_xc_lsda(wvlh_ctx *ctx, int64_t npts, const double *rho_up, const double *rho_dn, double *vxc_up,
                            double *vxc_dn, int accumulate, double dvol, double *energies)
{
    // each point's two densities are read before its potentials are written
    if (!ctx || npts < 0 || (npts > 0 && (!rho_up || !rho_dn || !vxc_up || !vxc_dn)) || vxc_up == vxc_dn)
        return ps_fail(WVLH_ERR_ARG);
    if (cudaSetDevice(ctx->device) != cudaSuccess) return ps_fail(WVLH_ERR_CUDA);
    if (npts == 0 && !energies) return WVLH_OK;
    PsPlan *pl;
    {
        std::lock_guard<std::mutex> lock(g_ps_mutex);
        const auto key = std::make_tuple((const void *)ctx, ctx->device, 0, 0, 0);
        auto it = g_ps_plans.find(key);
        if (it == g_ps_plans.end()) it = g_ps_plans.emplace(key, new PsPlan()).first;
        pl = it->second;
    }
    int rc = ps_energy_buffers(ctx, pl);
    if (rc) return ps_fail(rc);
    double *part = (double *)pl->part.p;
    unsigned int *cnt = (unsigned int *)pl->cnt.p;
    cudaStream_t st = ctx->stream;
    if (accumulate)
        k_xc_lsda<true><<<kPsBlocks, 256, 0, st>>>(npts, rho_up, rho_dn, vxc_up, vxc_dn, part, cnt, dvol, energies);
    else
        k_xc_lsda<false><<<kPsBlocks, 256, 0, st>>>(npts, rho_up, rho_dn, vxc_up, vxc_dn, part, cnt, dvol, energies);
    if (cudaGetLastError() != cudaSuccess) return ps_fail(WVLH_ERR_CUDA);
    return WVLH_OK;
}

static int ps_padded_hartree(wvlh_ctx *ctx, bool wire, const int n[3], const double h[3], const double *rho,
                             double *pot, double *eh, PsPlan **out);

// V_H into pot for boundary-condition code bc (0 periodic, offset 0; 1 free;
// 2 surface; 3 wire), no energy; returns the grid's plan for the energy partials
static int ps_hartree_bc(wvlh_ctx *ctx, int bc, const int n[3], const double h[3], const double *rho, double *pot,
                         PsPlan **pl)
{
    switch (bc) {
    case 0: return ps_hartree(ctx, n, h, rho, pot, 0.0, pl);
    case 1: return ps_free_hartree(ctx, n, h, rho, pot, nullptr, pl);
    case 2: return ps_padded_hartree(ctx, false, n, h, rho, pot, nullptr, pl);
    default: return ps_padded_hartree(ctx, true, n, h, rho, pot, nullptr, pl);
    }
}

extern "C" int wvlh_ks_potential_bc(wvlh_ctx *ctx, int bc, const int n[3], const double h[3], const double *rho,
                                    const double *rhocore, const double *vext, double *pot, double *energies)
{
    // the combine pass reads rho, the core density and V_ext after V_H is written to pot
    if (!ctx || !n || !h || !rho || !pot || pot == rho || (vext && vext == pot) || (rhocore && rhocore == pot) ||
        bc < 0 || bc > 3 ||
        (bc ? !ps_free_args_ok(n, h) : !ps_args_ok(n, h)))
        return ps_fail(WVLH_ERR_ARG);
    PsPlan *pl = nullptr;
    int rc = ps_hartree_bc(ctx, bc, n, h, rho, pot, &pl);
    if (rc) return ps_fail(rc);
    const long long npt = (long long)n[0] * n[1] * n[2];
    k_ks_combine<<<kPsBlocks, 256, 0, ctx->stream>>>(npt, rho, vext, pot, (double *)pl->part.p,
                                                     (unsigned int *)pl->cnt.p, h[0] * h[1] * h[2], energies, rhocore);
    if (cudaGetLastError() != cudaSuccess) return ps_fail(WVLH_ERR_CUDA);
    return WVLH_OK;
}

extern "C" int wvlh_ks_potential_spin(wvlh_ctx *ctx, int free_bc, const int n[3], const double h[3],
                                      const double *rho_up, const double *rho_dn, const double *rhocore,
                                      const double *vext, double *pot_up, double *pot_dn, double *energies)
{
    // pot_dn holds the total density for the Hartree solve, pot_up takes V_H:
    // neither may alias an input or the other
    if (!ctx || !n || !h || !rho_up || !rho_dn || !pot_up || !pot_dn || pot_up == pot_dn)
        return ps_fail(WVLH_ERR_ARG);
    for (const double *q : {rho_up, rho_dn, vext, rhocore})
        if (q && (q == pot_up || q == pot_dn)) return ps_fail(WVLH_ERR_ARG);
    if (free_bc < 0 || free_bc > 3 || (free_bc ? !ps_free_args_ok(n, h) : !ps_args_ok(n, h)))
        return ps_fail(WVLH_ERR_ARG);
    if (cudaSetDevice(ctx->device) != cudaSuccess) return ps_fail(WVLH_ERR_CUDA);
    const long long npt = (long long)n[0] * n[1] * n[2];
    k_spin_total<<<kPsBlocks, 256, 0, ctx->stream>>>(npt, rho_up, rho_dn, pot_dn);
    if (cudaGetLastError() != cudaSuccess) return ps_fail(WVLH_ERR_CUDA);
    PsPlan *pl = nullptr;
    int rc = ps_hartree_bc(ctx, free_bc, n, h, pot_dn, pot_up, &pl);
    if (rc) return ps_fail(rc);
    k_ks_combine_spin<<<kPsBlocks, 256, 0, ctx->stream>>>(npt, rho_up, rho_dn, vext, pot_up, pot_dn,
                                                          (double *)pl->part.p, (unsigned int *)pl->cnt.p,
                                                          h[0] * h[1] * h[2], energies, rhocore);
    if (cudaGetLastError() != cudaSuccess) return ps_fail(WVLH_ERR_CUDA);
    return WVLH_OK;
}

// the surface-BC plan of a grid (x, z periodic, y free): y padded to N2,
// cuFFT D2Z / Z2D over (n3, N2, n1), the kernel table (n3/2+1, N2/2+1,
// n1/2+1) built on the host once, the padded input (zero for y >= n2, set once)
static int ps_surface_plan(wvlh_ctx *ctx, const int n[3], const double h[3], PsPlan **out)
{
    std::lock_guard<std::mutex> lock(g_ps_mutex);
    const auto key = std::make_tuple((const void *)ctx, ctx->device, n[0], n[1], n[2], h[0], h[1], h[2]);
    auto it = g_ps_surf.find(key);
    if (it != g_ps_surf.end()) {
        *out = it->second;
        return WVLH_OK;
    }
    PsPlan *pl = new PsPlan();
    pl->nf[0] = n[0];
    pl->nf[1] = fft_length(2 * n[1]);
    pl->nf[2] = n[2];
    const int N1 = pl->nf[0], N2 = pl->nf[1], N3 = pl->nf[2];
    const size_t npad = (size_t)N3 * N2 * N1, nspec = (size_t)N3 * N2 * (N1 / 2 + 1);
    int rc = WVLH_OK;
    if (cufftPlan3d(&pl->fwd, N3, N2, N1, CUFFT_D2Z) != CUFFT_SUCCESS ||
        cufftPlan3d(&pl->inv, N3, N2, N1, CUFFT_Z2D) != CUFFT_SUCCESS)
        rc = WVLH_ERR_CUDA;
    std::vector<double> tab;
    if (!rc) {
        surface_kernel_table(n, h, N2, tab);
        if ((rc = pl->ker.ensure(sizeof(double) * tab.size())) || (rc = pl->pad.ensure(sizeof(double) * npad)) ||
            (rc = pl->work.ensure(sizeof(double) * npad)) ||
            (rc = pl->spec.ensure(sizeof(cufftDoubleComplex) * nspec)) || (rc = ps_energy_buffers(ctx, pl)))
            ;
    }
    if (!rc) {
        cudaStream_t st = ctx->stream;
        const bool ok =
            cudaMemcpyAsync(pl->ker.p, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice, st) ==
                cudaSuccess &&
            cudaMemsetAsync(pl->pad.p, 0, sizeof(double) * npad, st) == cudaSuccess &&
            cudaStreamSynchronize(st) == cudaSuccess;
        if (!ok) rc = WVLH_ERR_CUDA;
    }
    if (rc) {
        free_plan(pl);
        return rc;
    }
    g_ps_surf.emplace(key, pl);
    *out = pl;
    return WVLH_OK;
}

static int ps_wire_plan(wvlh_ctx *ctx, const int n[3], const double h[3], PsPlan **out);

// V_H of rho with surface (wire when wire) boundary conditions into pot; with
// eh, *eh = the Hartree energy (reduced by the crop)
static int ps_padded_hartree(wvlh_ctx *ctx, bool wire, const int n[3], const double h[3], const double *rho,
                             double *pot, double *eh, PsPlan **out)
{
    if (cudaSetDevice(ctx->device) != cudaSuccess) return WVLH_ERR_CUDA;
    PsPlan *pl = nullptr;
    int rc = wire ? ps_wire_plan(ctx, n, h, &pl) : ps_surface_plan(ctx, n, h, &pl);
    if (rc) return rc;
    const int N1 = pl->nf[0], N2 = pl->nf[1], N3 = pl->nf[2];
    cudaStream_t st = ctx->stream;
    double *pad = (double *)pl->pad.p, *work = (double *)pl->work.p;
    cufftDoubleComplex *z = (cufftDoubleComplex *)pl->spec.p;
    k_free_pad<<<kPsBlocks, 256, 0, st>>>(n[0], n[1], n[2], N1, N2, rho, pad);
    bool ok = cudaGetLastError() == cudaSuccess && cufftSetStream(pl->fwd, st) == CUFFT_SUCCESS &&
              cufftSetStream(pl->inv, st) == CUFFT_SUCCESS && cufftExecD2Z(pl->fwd, pad, z) == CUFFT_SUCCESS;
    if (ok) {
        // surface: -4 pi h_y / (N1 N2 N3), createKernel.f90:374; wire: -2 h_x h_y / (N1 N2 N3), :502
        const double scal = (wire ? -2.0 * h[0] * h[1] : -4.0 * 3.14159265358979323846 * h[1]) /
                            ((double)N1 * (double)N2 * (double)N3);
        k_table_multiply<<<kPsBlocks, 256, 0, st>>>(N1, N2, N3, (const double *)pl->ker.p, scal, 0, 0.0, z);
        ok = cudaGetLastError() == cudaSuccess && cufftExecZ2D(pl->inv, z, work) == CUFFT_SUCCESS;
    }
    if (ok) {
        k_free_crop<<<kPsBlocks, 256, 0, st>>>(n[0], n[1], n[2], N1, N2, work, rho, pot, (double *)pl->part.p,
                                               (unsigned int *)pl->cnt.p, 0.5 * h[0] * h[1] * h[2], eh);
        ok = cudaGetLastError() == cudaSuccess;
    }
    if (!ok) return WVLH_ERR_CUDA;
    *out = pl;
    return WVLH_OK;
}

extern "C" int wvlh_psolver_surface(wvlh_ctx *ctx, const int n[3], const double h[3], const double *rho,
                                    double *pot, double *eh)
{
    // rho is copied into the padded buffer before pot is written: pot may be
    // rho, unless the energy (which reads rho after) is asked for
    if (!ctx || !n || !h || !rho || !pot || (eh && pot == rho) || !ps_free_args_ok(n, h))
        return ps_fail(WVLH_ERR_ARG);
    PsPlan *pl = nullptr;
    const int rc = ps_padded_hartree(ctx, false, n, h, rho, pot, eh, &pl);
    return rc ? ps_fail(rc) : WVLH_OK;
}

extern "C" int64_t wvlh_psolver_surface_table(const int n[3], const double h[3], int *N2, double *tab, int64_t cap)
{
    if (!n || !h || !N2 || !ps_free_args_ok(n, h)) return -(int64_t)ps_fail(WVLH_ERR_ARG);
    *N2 = fft_length(2 * n[1]);
    const int64_t need = (int64_t)(n[2] / 2 + 1) * (*N2 / 2 + 1) * (n[0] / 2 + 1);
    if (!tab) return need;
    if (cap < need) return -(int64_t)ps_fail(WVLH_ERR_ARG);
    std::vector<double> t;
    surface_kernel_table(n, h, *N2, t);
    std::copy(t.begin(), t.end(), tab);
    return need;
}

// the wire-BC plan of a grid (z periodic, x and y free): x and y padded,
// cuFFT D2Z / Z2D over (n_z, Ny, Nx), the kernel table built on the host once,
// the padded input (zero outside the (n_y, n_x) corner, set once)
static int ps_wire_plan(wvlh_ctx *ctx, const int n[3], const double h[3], PsPlan **out)
{
    std::lock_guard<std::mutex> lock(g_ps_mutex);
    const auto key = std::make_tuple((const void *)ctx, ctx->device, n[0], n[1], n[2], h[0], h[1], h[2]);
    auto it = g_ps_wire.find(key);
    if (it != g_ps_wire.end()) {
        *out = it->second;
        return WVLH_OK;
    }
    PsPlan *pl = new PsPlan();
    pl->nf[0] = fft_length(2 * n[0]);
    pl->nf[1] = fft_length(2 * n[1]);
    pl->nf[2] = n[2];
    const int N1 = pl->nf[0], N2 = pl->nf[1], N3 = pl->nf[2];
    const size_t npad = (size_t)N3 * N2 * N1, nspec = (size_t)N3 * N2 * (N1 / 2 + 1);
    int rc = WVLH_OK;
    if (cufftPlan3d(&pl->fwd, N3, N2, N1, CUFFT_D2Z) != CUFFT_SUCCESS ||
        cufftPlan3d(&pl->inv, N3, N2, N1, CUFFT_Z2D) != CUFFT_SUCCESS)
        rc = WVLH_ERR_CUDA;
    std::vector<double> tab;
    if (!rc) {
        wire_kernel_table(n, h, N1, N2, tab);
        if ((rc = pl->ker.ensure(sizeof(double) * tab.size())) || (rc = pl->pad.ensure(sizeof(double) * npad)) ||
            (rc = pl->work.ensure(sizeof(double) * npad)) ||
            (rc = pl->spec.ensure(sizeof(cufftDoubleComplex) * nspec)) || (rc = ps_energy_buffers(ctx, pl)))
            ;
    }
    if (!rc) {
        cudaStream_t st = ctx->stream;
        const bool ok =
            cudaMemcpyAsync(pl->ker.p, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice, st) ==
                cudaSuccess &&
            cudaMemsetAsync(pl->pad.p, 0, sizeof(double) * npad, st) == cudaSuccess &&
            cudaStreamSynchronize(st) == cudaSuccess;
        if (!ok) rc = WVLH_ERR_CUDA;
    }
    if (rc) {
        free_plan(pl);
        return rc;
    }
    g_ps_wire.emplace(key, pl);
    *out = pl;
    return WVLH_OK;
}

extern "C" int wvlh_psolver_wire(wvlh_ctx *ctx, const int n[3], const double h[3], const double *rho, double *pot,
                                 double *eh)
{
    if (!ctx || !n || !h || !rho || !pot || (eh && pot == rho) || !ps_free_args_ok(n, h))
        return ps_fail(WVLH_ERR_ARG);
    PsPlan *pl = nullptr;
    const int rc = ps_padded_hartree(ctx, true, n, h, rho, pot, eh, &pl);
    return rc ? ps_fail(rc) : WVLH_OK;
}

extern "C" int64_t wvlh_psolver_wire_table(const int n[3], const double h[3], int nf[2], double *tab, int64_t cap)
{
    if (!n || !h || !nf || !ps_free_args_ok(n, h)) return -(int64_t)ps_fail(WVLH_ERR_ARG);
    nf[0] = fft_length(2 * n[0]);
    nf[1] = fft_length(2 * n[1]);
    const int64_t need = (int64_t)(n[2] / 2 + 1) * (nf[1] / 2 + 1) * (nf[0] / 2 + 1);
    if (!tab) return need;
    if (cap < need) return -(int64_t)ps_fail(WVLH_ERR_ARG);
    std::vector<double> t;
    wire_kernel_table(n, h, nf[0], nf[1], t);
    std::copy(t.begin(), t.end(), tab);
    return need;
}
