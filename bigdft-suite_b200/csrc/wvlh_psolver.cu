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

struct PsPlan {
    cufftHandle fwd = 0, inv = 0;
    DevBuf spec, fac, part;
};

}  // namespace wvlh

using namespace wvlh;

// plans and buffers per (context, device, grid), kept for the process: an SCF
// loop solves on the same grid at every iteration
static std::mutex g_ps_mutex;
static std::map<std::tuple<const void *, int, int, int, int>, PsPlan *> g_ps_plans;

extern "C" int wvlh_psolver_periodic(wvlh_ctx *ctx, const int n[3], const double h[3], const double *rho,
                                     double *pot, double offset, double *eh)
{
    // the energy needs rho after the potential is written: no aliasing then
    if (!ctx || !n || !h || !rho || !pot || (eh && pot == rho)) {
        set_last_error(WVLH_ERR_ARG);
        return WVLH_ERR_ARG;
    }
    for (int k = 0; k < 3; ++k)
        if (n[k] < 16 || n[k] % 2 || !(h[k] > 0.0)) {   // the ISF needs 16 points, the kernel even sizes
            set_last_error(WVLH_ERR_ARG);
            return WVLH_ERR_ARG;
        }
    if (cudaSetDevice(ctx->device) != cudaSuccess) {
        set_last_error(WVLH_ERR_CUDA);
        return WVLH_ERR_CUDA;
    }
    const int n1 = n[0], n2 = n[1], n3 = n[2];
    const long long npt = (long long)n1 * n2 * n3, nc = (long long)n3 * n2 * (n1 / 2 + 1);
    PsPlan *pl;
    {
        std::lock_guard<std::mutex> lock(g_ps_mutex);
        const auto key = std::make_tuple((const void *)ctx, ctx->device, n1, n2, n3);
        auto it = g_ps_plans.find(key);
        if (it == g_ps_plans.end()) {
            // cuFFT's last dimension is the fastest: (n3, n2, n1) for x-fastest arrays
            cufftHandle f = 0, b = 0;
            if (cufftPlan3d(&f, n3, n2, n1, CUFFT_D2Z) != CUFFT_SUCCESS) {
                set_last_error(WVLH_ERR_CUDA);
                return WVLH_ERR_CUDA;
            }
            if (cufftPlan3d(&b, n3, n2, n1, CUFFT_Z2D) != CUFFT_SUCCESS) {
                cufftDestroy(f);
                set_last_error(WVLH_ERR_CUDA);
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
    const int nblk = 1184;   // 8 per SM on 148 SMs
    if ((rc = pl->spec.ensure(sizeof(cufftDoubleComplex) * (size_t)nc)) ||
        (rc = pl->fac.ensure(sizeof(double) * (size_t)(n1 / 2 + n2 / 2 + n3 / 2 + 3))) ||
        (rc = pl->part.ensure(sizeof(double) * (size_t)(nblk + 1)))) {
        set_last_error(rc);
        return rc;
    }
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
        k_ps_multiply<<<nblk, 256, 0, st>>>(n1, n2, n3, n1 * h[0], n2 * h[1], n3 * h[2], d_fac, d_fac + fx.size(),
                                            d_fac + fx.size() + fy.size(), scal, offset / vol * scal, z);
        ok = cudaGetLastError() == cudaSuccess;
    }
    if (ok) ok = cufftExecZ2D(pl->inv, z, (cufftDoubleReal *)pot) == CUFFT_SUCCESS;
    if (ok && eh) {
        double *part = (double *)pl->part.p;
        k_ps_dot<<<nblk, 256, 0, st>>>(npt, rho, pot, part);
        k_ps_sum<<<1, 1024, 0, st>>>(nblk, part, 0.5 * vol, eh);
        ok = cudaGetLastError() == cudaSuccess;
    }
    if (!ok) {
        set_last_error(WVLH_ERR_CUDA);
        return WVLH_ERR_CUDA;
    }
    return WVLH_OK;
}
