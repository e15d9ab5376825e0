// Host launchers of the plain per-pass kernels (wvlh_plain.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace wvlh {

// Rotated 1D passes, OpenCL layout in[p*ndat+j] -> out[j*Lout+q]; nb batches
// at element strides bi (input) / bo (output).
cudaError_t plain_syn1d(int N, int ndat, int per, const double *in, double *out, int nb, size_t bi, size_t bo,
                        cudaStream_t st);
cudaError_t plain_ana1d(int N, int ndat, int per, const double *in, double *out, int nb, size_t bi, size_t bo,
                        cudaStream_t st);
// mode 0 mf periodic, 1 mf^T periodic, 2 mf grow (n -> n+15), 3 mf^T shrink (n+15 -> n)
cudaError_t plain_mf1d(int mode, int n, int ndat, const double *in, double *out, int nb, size_t bi, size_t bo,
                       cudaStream_t st);
cudaError_t plain_kin1d(int n, int ndat, int per, double scale, const double *x_in, double *x_out,
                        const double *y_in, double *y_out, int nb, size_t bi, size_t bo, cudaStream_t st);
// dir 0 uncompress (zeroes psig first), 1 compress; scal_host: 8 scale factors (host) or null
cudaError_t plain_uncompress(int dir, const int *dims, int nseg_c, int nvctr_c, const uint32_t *keyg_c,
                             const uint32_t *keyv_c, int nseg_f, int nvctr_f, const uint32_t *keyg_f,
                             const uint32_t *keyv_f, double *psi_c, double *psi_f, double *psig,
                             const double *scal_host, int nb, size_t bpsi_c, size_t bpsi_f, size_t bpsig,
                             cudaStream_t st);
cudaError_t plain_potential(size_t n, const double *pot, double *psir, double *part, int nparts, double *epot_dev,
                            cudaStream_t st);
cudaError_t plain_axpy(size_t n, double alpha, const double *x, const double *y, double *z, cudaStream_t st);
cudaError_t plain_scal(size_t n, double alpha, const double *x, double *y, cudaStream_t st);
cudaError_t plain_set(size_t n, double v, double *x, cudaStream_t st);
cudaError_t plain_square_axpy(size_t n, double alpha, const double *x, double *y, cudaStream_t st);
cudaError_t plain_dot(size_t n, const double *x, const double *y, double *part, double *out_dev, cudaStream_t st);
cudaError_t plain_square(size_t n, double *x, cudaStream_t st);
cudaError_t plain_scale7(size_t nvf, const double *s7, double *psi_f, cudaStream_t st);

constexpr int kDotParts = 1184;

}  // namespace wvlh
