// Plain (one kernel per 1D pass) operators with the data layouts of the
// reference's OpenCL backend, behind the per-op ocl_* entry points.
//
// Layout conventions (bigdft/src/OpenCL/Wavelet.c, MagicFilter.c, Kinetic.c):
// a 1D pass over n positions and ndat lines reads in[p*ndat + j] and writes
// the rotated out[j*Lout + q]; three passes over z, y, x return a 3D array to
// its natural x-fastest layout.  Compressed vectors use 1-based uint32 keys
// keyg(2,nseg)/keyv(nseg) and the segment of an element is found by binary
// search on keyv, as the OpenCL (un)compress kernels do
// (OpenCL/Uncompress.c:17-80).
#include <cuda_runtime.h>

#include "wvlh_common.cuh"
#include "wvlh_plain.h"

namespace wvlh {

constexpr int JT = 32;  // lines per CTA in the rotated passes

enum PassKind { P_SYN = 0, P_ANA, P_MF, P_MFT, P_MFG, P_MFS, P_KIN };

// Rotated 1D pass.  For P_SYN/P_ANA, n is the coarse count N and `per`
// selects periodic or grow/shrink; for the MF family n is the input length;
// for P_KIN n is the line length and the pass also rotates x (x_out) and
// adds y_in (y_out = y_in + scale*K x), like OpenCL kinetic1dKernel_d.
template <int KIND>
__global__ void __launch_bounds__(256) k_pass1d(int n, int ndat, int per, double scale, const double *__restrict__ in,
                                                 double *__restrict__ out, const double *__restrict__ yin,
                                                 double *__restrict__ xout, size_t batch_in, size_t batch_out)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    int Lin, Lout;
    if (KIND == P_SYN) { Lin = 2 * n; Lout = fine_len(n, per); }
    else if (KIND == P_ANA) { Lin = fine_len(n, per); Lout = 2 * n; }
    else if (KIND == P_MFG) { Lin = n; Lout = n + 15; }
    else if (KIND == P_MFS) { Lin = n + 15; Lout = n; }
    else { Lin = n; Lout = n; }
    const int Lp = Lout | 1;
    double *S = reinterpret_cast<double *>(smem_raw);   // [Lin][JT+1]
    double *D = S + (size_t)Lin * (JT + 1);             // [JT][Lp]
    const int j0 = blockIdx.x * JT;
    const double *gin = in + blockIdx.y * batch_in;
    double *gout = out + blockIdx.y * batch_out;
    for (int i = threadIdx.x; i < Lin * JT; i += blockDim.x) {
        const int p = i / JT, jj = i - p * JT;
        const int j = j0 + jj;
        S[p * (JT + 1) + jj] = (j < ndat) ? gin[(size_t)p * ndat + j] : 0.0;
    }
    __syncthreads();
    const LineGeom g{JT, 1, JT + 1, Lp, 1};
    double e = 0.0;
    if (KIND == P_SYN) pass_syn<double, 4>(S, D, g, n, n, per);
    else if (KIND == P_ANA) pass_ana<double, 4>(S, D, g, n, n, per);
    else if (KIND == P_MF) pass_mf<double, 4, 0>(S, D, g, Lin, Lout);
    else if (KIND == P_MFT) pass_mf<double, 4, 1>(S, D, g, Lin, Lout);
    else if (KIND == P_MFG) pass_mf<double, 4, 2>(S, D, g, Lin, Lout);
    else if (KIND == P_MFS) pass_mf<double, 4, 3>(S, D, g, Lin, Lout);
    else pass_kin<double, 4, false>(S, D, g, n, per, scale, 0.0, &e);
    __syncthreads();
    for (int i = threadIdx.x; i < Lout * JT; i += blockDim.x) {
        const int jj = i / Lout, q = i - jj * Lout;
        const int j = j0 + jj;
        if (j < ndat) {
            double v = D[jj * Lp + q];
            if (KIND == P_KIN) {
                v += yin[blockIdx.y * batch_in + (size_t)q * ndat + j];
                xout[blockIdx.y * batch_out + (size_t)j * Lout + q] = S[q * (JT + 1) + jj];
            }
            gout[(size_t)j * Lout + q] = v;
        }
    }
}

template <int KIND>
static cudaError_t pass1d(int n, int ndat, int per, double scale, const double *in, double *out, const double *yin,
                          double *xout, int nbatch, size_t batch_in, size_t batch_out, cudaStream_t st)
{
    int Lin, Lout;
    if (KIND == P_SYN) { Lin = 2 * n; Lout = fine_len(n, per); }
    else if (KIND == P_ANA) { Lin = fine_len(n, per); Lout = 2 * n; }
    else if (KIND == P_MFG) { Lin = n; Lout = n + 15; }
    else if (KIND == P_MFS) { Lin = n + 15; Lout = n; }
    else { Lin = n; Lout = n; }
    const size_t smem = ((size_t)Lin * (JT + 1) + (size_t)JT * (Lout | 1)) * sizeof(double);
    cudaError_t err = cudaFuncSetAttribute(k_pass1d<KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    dim3 grid((ndat + JT - 1) / JT, nbatch);
    k_pass1d<KIND><<<grid, 256, smem, st>>>(n, ndat, per, scale, in, out, yin, xout, batch_in, batch_out);
    return cudaGetLastError();
}

cudaError_t plain_syn1d(int N, int ndat, int per, const double *in, double *out, int nb, size_t bi, size_t bo,
                        cudaStream_t st)
{
    return pass1d<P_SYN>(N, ndat, per, 0.0, in, out, nullptr, nullptr, nb, bi, bo, st);
}
cudaError_t plain_ana1d(int N, int ndat, int per, const double *in, double *out, int nb, size_t bi, size_t bo,
                        cudaStream_t st)
{
    return pass1d<P_ANA>(N, ndat, per, 0.0, in, out, nullptr, nullptr, nb, bi, bo, st);
}
cudaError_t plain_mf1d(int mode, int n, int ndat, const double *in, double *out, int nb, size_t bi, size_t bo,
                       cudaStream_t st)
{
    switch (mode) {
    case 0: return pass1d<P_MF>(n, ndat, 1, 0.0, in, out, nullptr, nullptr, nb, bi, bo, st);
    case 1: return pass1d<P_MFT>(n, ndat, 1, 0.0, in, out, nullptr, nullptr, nb, bi, bo, st);
    case 2: return pass1d<P_MFG>(n, ndat, 0, 0.0, in, out, nullptr, nullptr, nb, bi, bo, st);
    default: return pass1d<P_MFS>(n, ndat, 0, 0.0, in, out, nullptr, nullptr, nb, bi, bo, st);
    }
}
cudaError_t plain_kin1d(int n, int ndat, int per, double scale, const double *x_in, double *x_out,
                        const double *y_in, double *y_out, int nb, size_t bi, size_t bo, cudaStream_t st)
{
    return pass1d<P_KIN>(n, ndat, per, scale, x_in, y_out, y_in, x_out, nb, bi, bo, st);
}

// ---------------------------------------------------------------- (un)compress
__device__ __forceinline__ int find_seg(const uint32_t *keyv, int nseg, int ig)
{
    // largest iseg with keyv[iseg]-1 <= ig (OpenCL/Uncompress.c:24-38)
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if ((int)keyv[mid] - 1 <= ig) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// psi_g index of (i1,s1,i2,s2,i3,s3) with n1,n2,n3 coarse counts
__device__ __forceinline__ size_t gpos(int n1, int n2, int n3, int i1, int s1, int i2, int s2, int i3, int s3)
{
    return ((((size_t)s3 * n3 + i3) * 2 + s2) * n2 + i2) * 2 * (size_t)n1 + (size_t)s1 * n1 + i1;
}

// dir 0: uncompress (psi -> psi_g), dir 1: compress (psi_g -> psi)
struct Scal8 {
    double s[8];
};

template <int DIR, bool FINE>
__global__ void k_uncompress(int n1, int n2, int n3, int nseg, int nvctr, const uint32_t *__restrict__ keyg,
                             const uint32_t *__restrict__ keyv, double *__restrict__ psi, double *__restrict__ psig,
                             const Scal8 sc, int use_scal, size_t bpsi, size_t bpsig)
{
    const int ig = blockIdx.x * blockDim.x + threadIdx.x;
    if (ig >= nvctr) return;
    psi += blockIdx.y * bpsi;
    psig += blockIdx.y * bpsig;
    const int iseg = find_seg(keyv, nseg, ig);
    const int j0 = (int)keyg[2 * iseg];
    int ii = j0 - 1;
    const int i3 = ii / (n1 * n2);
    ii -= i3 * n1 * n2;
    const int i2 = ii / n1;
    const int i1 = ii - i2 * n1 + ig - ((int)keyv[iseg] - 1);
    // caller keys are not validated on this path (as in the reference): never
    // touch memory outside the box for malformed keys
    if (j0 < 1 || (unsigned)i1 >= (unsigned)n1 || (unsigned)i2 >= (unsigned)n2 || (unsigned)i3 >= (unsigned)n3)
        return;
    if (!FINE) {
        const size_t p = gpos(n1, n2, n3, i1, 0, i2, 0, i3, 0);
        const double s = use_scal ? sc.s[0] : 1.0;
        if (DIR == 0) psig[p] = psi[ig] * s; else psi[ig] = psig[p] * s;
    } else {
#pragma unroll
        for (int c = 1; c <= 7; ++c) {
            const size_t p = gpos(n1, n2, n3, i1, c & 1, i2, (c >> 1) & 1, i3, (c >> 2) & 1);
            const double s = use_scal ? sc.s[c] : 1.0;
            if (DIR == 0) psig[p] = psi[7 * (size_t)ig + c - 1] * s;
            else psi[7 * (size_t)ig + c - 1] = psig[p] * s;
        }
    }
}

cudaError_t plain_uncompress(int dir, const int *dims, int nseg_c, int nvctr_c, const uint32_t *keyg_c,
                             const uint32_t *keyv_c, int nseg_f, int nvctr_f, const uint32_t *keyg_f,
                             const uint32_t *keyv_f, double *psi_c, double *psi_f, double *psig,
                             const double *scal_host, int nb, size_t bpsi_c, size_t bpsi_f, size_t bpsig,
                             cudaStream_t st)
{
    const int n1 = dims[0], n2 = dims[1], n3 = dims[2];
    Scal8 sc;
    const int us = scal_host != nullptr;
    for (int k = 0; k < 8; ++k) sc.s[k] = us ? scal_host[k] : 1.0;
    if (dir == 0) {
        for (int b = 0; b < nb; ++b)
            cudaMemsetAsync(psig + b * bpsig, 0, sizeof(double) * 8 * (size_t)n1 * n2 * n3, st);
    }
    if (nvctr_c > 0) {
        dim3 g((nvctr_c + 255) / 256, nb);
        if (dir == 0)
            k_uncompress<0, false><<<g, 256, 0, st>>>(n1, n2, n3, nseg_c, nvctr_c, keyg_c, keyv_c, psi_c, psig,
                                                      sc, us, bpsi_c, bpsig);
        else
            k_uncompress<1, false><<<g, 256, 0, st>>>(n1, n2, n3, nseg_c, nvctr_c, keyg_c, keyv_c, psi_c, psig,
                                                      sc, us, bpsi_c, bpsig);
    }
    if (nvctr_f > 0) {
        dim3 g((nvctr_f + 255) / 256, nb);
        if (dir == 0)
            k_uncompress<0, true><<<g, 256, 0, st>>>(n1, n2, n3, nseg_f, nvctr_f, keyg_f, keyv_f, psi_f, psig, sc,
                                                     us, bpsi_f, bpsig);
        else
            k_uncompress<1, true><<<g, 256, 0, st>>>(n1, n2, n3, nseg_f, nvctr_f, keyg_f, keyv_f, psi_f, psig, sc,
                                                     us, bpsi_f, bpsig);
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------- elementwise / BLAS-1
__global__ void k_potential(size_t n, const double *__restrict__ pot, double *__restrict__ psir,
                            double *__restrict__ part, size_t bpsi)
{
    __shared__ double red[32];
    psir += blockIdx.y * bpsi;
    double e = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double r = psir[i];
        const double w = pot[i] * r;
        e += w * r;
        psir[i] = w;
    }
    const double s = block_sum(e, red);
    if (threadIdx.x == 0 && part) part[blockIdx.y * gridDim.x + blockIdx.x] = s;
}

// z = alpha*x + y  (and in-place forms); dot partials; all deterministic
__global__ void k_axpy(size_t n, double alpha, const double *x, const double *y, double *z)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        z[i] = alpha * x[i] + y[i];
}
__global__ void k_scal(size_t n, double alpha, const double *x, double *y)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] = alpha * x[i];
}
__global__ void k_set(size_t n, double v, double *x)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        x[i] = v;
}
__global__ void k_square_axpy(size_t n, double alpha, const double *x, double *y)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] += alpha * x[i] * x[i];
}
__global__ void k_dot_part(size_t n, const double *__restrict__ x, const double *__restrict__ y,
                           double *__restrict__ part)
{
    __shared__ double red[32];
    double e = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        e += x[i] * y[i];
    const double s = block_sum(e, red);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}
__global__ void k_sum_parts(int n, const double *__restrict__ part, double *__restrict__ out)
{
    __shared__ double red[32];
    double e = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) e += part[i];
    const double s = block_sum(e, red);
    if (threadIdx.x == 0) *out = s;
}

__global__ void k_square(size_t n, double *x)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        x[i] = x[i] * x[i];
}
// psi_f(7, nvf) *= s[0..6] per component (OpenCL scale_psi_fineKernel_d)
__global__ void k_scale7(size_t nvf, Scal8 sc, double *psi_f)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < 7 * nvf; i += (size_t)gridDim.x * blockDim.x)
        psi_f[i] *= sc.s[i % 7];
}

static inline int nblk(size_t n) { return (int)((n + 255) / 256 < 1184 ? (n + 255) / 256 : 1184); }

cudaError_t plain_square(size_t n, double *x, cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    k_square<<<nblk(n), 256, 0, st>>>(n, x);
    return cudaGetLastError();
}
cudaError_t plain_scale7(size_t nvf, const double *s7, double *psi_f, cudaStream_t st)
{
    if (nvf == 0) return cudaSuccess;
    Scal8 sc;
    for (int k = 0; k < 7; ++k) sc.s[k] = s7[k];
    sc.s[7] = 0.0;
    k_scale7<<<nblk(7 * nvf), 256, 0, st>>>(nvf, sc, psi_f);
    return cudaGetLastError();
}

cudaError_t plain_potential(size_t n, const double *pot, double *psir, double *part, int nparts, double *epot_dev,
                            cudaStream_t st)
{
    dim3 g(nparts, 1);
    k_potential<<<g, 256, 0, st>>>(n, pot, psir, part, 0);
    if (epot_dev) k_sum_parts<<<1, 256, 0, st>>>(nparts, part, epot_dev);
    return cudaGetLastError();
}

cudaError_t plain_axpy(size_t n, double alpha, const double *x, const double *y, double *z, cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    k_axpy<<<nblk(n), 256, 0, st>>>(n, alpha, x, y, z);
    return cudaGetLastError();
}
cudaError_t plain_scal(size_t n, double alpha, const double *x, double *y, cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    k_scal<<<nblk(n), 256, 0, st>>>(n, alpha, x, y);
    return cudaGetLastError();
}
cudaError_t plain_set(size_t n, double v, double *x, cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    k_set<<<nblk(n), 256, 0, st>>>(n, v, x);
    return cudaGetLastError();
}
cudaError_t plain_square_axpy(size_t n, double alpha, const double *x, double *y, cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    k_square_axpy<<<nblk(n), 256, 0, st>>>(n, alpha, x, y);
    return cudaGetLastError();
}
// part must hold 1184 doubles; the result lands in *out_dev
cudaError_t plain_dot(size_t n, const double *x, const double *y, double *part, double *out_dev, cudaStream_t st)
{
    if (n == 0) return cudaMemsetAsync(out_dev, 0, sizeof(double), st);
    const int nb = nblk(n);
    k_dot_part<<<nb, 256, 0, st>>>(n, x, y, part);
    k_sum_parts<<<1, 256, 0, st>>>(nb, part, out_dev);
    return cudaGetLastError();
}

}  // namespace wvlh
