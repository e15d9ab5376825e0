/*
 * wvlh — B200-native Daubechies-16 wavelet local Hamiltonian.
 *
 * C ABI.  Two groups of entry points:
 *
 *  1. Drop-in replacements for the accelerator wrappers BigDFT's Fortran host
 *     already calls (bigdft/src/OpenCL/OpenCL_wrappers.h, FC_FUNC_ mangling:
 *     lower case + trailing underscore, every argument by pointer).  Buffers
 *     (cl_mem) are opaque handles to device allocations owned by the caller,
 *     exactly as in the reference (interface_ocl.f90:43-190 allocates, :196-260
 *     frees).  Keys are device buffers of 1-based uint32 keyg(2,nseg)/keyv(nseg).
 *     Errors never exit(): they are recorded on the queue (sticky) and in a
 *     process-wide slot read by wvlh_get_last_error().  Only the Gamma point
 *     (nspinor == 1) is supported by the *_k entry points; nspinor == 2 records
 *     WVLH_ERR_UNSUPPORTED.
 *
 *  2. New batched entry points (wvlh_*): many orbitals and many localisation
 *     regions per call, FP32 or FP64 compute, device pointers, returning an
 *     int status (0 = success).
 *
 * All FP64 results match the reference's CPU convolutions within 1e-13
 * relative L2; FP32 forms keep energies, densities and scalar products in FP64.
 */
#ifndef WVLH_H
#define WVLH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef uint32_t cl_uint;
typedef int32_t cl_int;
typedef double cl_double;
typedef struct wvlh_mem *cl_mem;
typedef struct wvlh_ocl_context *bigdft_context;
typedef struct wvlh_ocl_queue *bigdft_command_queue;

enum {
    WVLH_OK = 0,
    WVLH_ERR_CUDA = 1,
    WVLH_ERR_ARG = 2,
    WVLH_ERR_KEYS = 3,
    WVLH_ERR_NOMEM = 4,
    WVLH_ERR_UNSUPPORTED = 5,
    WVLH_ERR_TOO_LARGE = 6,
    WVLH_ERR_STALE = 7
};

/* --------------------------------------------------------------------- */
/* 1. drop-in OpenCL-wrapper ABI                                          */
/* --------------------------------------------------------------------- */

/* lifecycle: OpenCL_wrappers.h:309-381 */
void ocl_create_context_(bigdft_context *context, const char *platform, const char *devices, cl_int *device_type,
                         cl_uint *device_number);                                       /* :315 */
void ocl_create_gpu_context_(bigdft_context *context, cl_uint *device_number);         /* :317 */
void ocl_build_programs_(bigdft_context *context);                                     /* :313 */
void ocl_create_command_queue_(bigdft_command_queue *command_queue, bigdft_context *context); /* :370 */
void ocl_create_command_queue_id_(bigdft_command_queue *command_queue, bigdft_context *context,
                                  cl_uint *index);                                     /* :372 */
void ocl_create_read_buffer_(bigdft_context *context, cl_uint *size, cl_mem *buff_ptr);        /* :325 */
void ocl_create_write_buffer_(bigdft_context *context, cl_uint *size, cl_mem *buff_ptr);       /* :338 */
void ocl_create_read_write_buffer_(bigdft_context *context, cl_uint *size, cl_mem *buff_ptr);  /* :331 */
void ocl_create_read_buffer_and_copy_(bigdft_context *context, cl_uint *size, void *host_ptr,
                                      cl_mem *buff_ptr);                               /* :332 */
void ocl_release_mem_object_(cl_mem *buff_ptr);                                         /* :340 */
/* Buffers over caller host memory (CL_MEM_USE_HOST_PTR) and pinned regions,
   OpenCL_wrappers.h:1238-1253 (bodies OpenCL_wrappers.c:345-505): the range is
   page-locked (cudaHostRegister, mapped) so queued copies to and from it are
   DMA transfers; releasing the handle unlocks the range once the copies queued
   before the release are done.  A map makes the host memory current after the
   commands queued before it (blocking forms wait for the queue; asynchronous
   forms and unmap are queue-ordered and need no work). */
void ocl_create_read_buffer_host_(bigdft_context *context, cl_uint *size, void *host_ptr, cl_mem *buff_ptr); /* :1238 */
void ocl_create_write_buffer_host_(bigdft_context *context, cl_uint *size, void *host_ptr, cl_mem *buff_ptr); /* :1239 */
void ocl_create_read_write_buffer_host_(bigdft_context *context, cl_uint *size, void *host_ptr,
                                        cl_mem *buff_ptr);                             /* :1240 */
void ocl_map_read_buffer_(bigdft_command_queue *command_queue, cl_mem *buff_ptr, cl_uint *offset,
                          cl_uint *size);                                              /* :1241 */
void ocl_map_write_buffer_(bigdft_command_queue *command_queue, cl_mem *buff_ptr, cl_uint *offset,
                           cl_uint *size);                                             /* :1242 */
void ocl_map_read_write_buffer_(bigdft_command_queue *command_queue, cl_mem *buff_ptr, cl_uint *offset,
                                cl_uint *size);                                        /* :1243 */
void ocl_map_read_buffer_async_(bigdft_command_queue *command_queue, cl_mem *buff_ptr, cl_uint *offset,
                                cl_uint *size);                                        /* :1244 */
void ocl_map_write_buffer_async_(bigdft_command_queue *command_queue, cl_mem *buff_ptr, cl_uint *offset,
                                 cl_uint *size);                                       /* :1245 */
void ocl_map_read_write_buffer_async_(bigdft_command_queue *command_queue, cl_mem *buff_ptr, cl_uint *offset,
                                      cl_uint *size);                                  /* :1246 */
void ocl_unmap_mem_object_(bigdft_command_queue *command_queue, cl_mem *buff_ptr, void *host_ptr); /* :1247 */
void ocl_pin_read_write_buffer_(bigdft_context *context, bigdft_command_queue *command_queue, cl_uint *size,
                                void *host_ptr, cl_mem *buff_ptr);                     /* :1248 */
void ocl_pin_write_buffer_(bigdft_context *context, bigdft_command_queue *command_queue, cl_uint *size,
                           void *host_ptr, cl_mem *buff_ptr);                          /* :1249 */
void ocl_pin_read_buffer_(bigdft_context *context, bigdft_command_queue *command_queue, cl_uint *size,
                          void *host_ptr, cl_mem *buff_ptr);                           /* :1250 */
void ocl_pin_read_write_buffer_async_(bigdft_context *context, bigdft_command_queue *command_queue, cl_uint *size,
                                      void *host_ptr, cl_mem *buff_ptr);               /* :1251 */
void ocl_pin_write_buffer_async_(bigdft_context *context, bigdft_command_queue *command_queue, cl_uint *size,
                                 void *host_ptr, cl_mem *buff_ptr);                    /* :1252 */
void ocl_pin_read_buffer_async_(bigdft_context *context, bigdft_command_queue *command_queue, cl_uint *size,
                                void *host_ptr, cl_mem *buff_ptr);                     /* :1253 */
void ocl_enqueue_read_buffer_(bigdft_command_queue *command_queue, cl_mem *buffer, cl_uint *size,
                              void *host_ptr);                                         /* :347 */
void ocl_enqueue_write_buffer_(bigdft_command_queue *command_queue, cl_mem *buffer, cl_uint *size,
                               const void *host_ptr);                                  /* :354 */
void ocl_enqueue_read_buffer_async_(bigdft_command_queue *command_queue, cl_mem *buffer, cl_uint *size,
                                    void *host_ptr);                                   /* :361 */
void ocl_enqueue_write_buffer_async_(bigdft_command_queue *command_queue, cl_mem *buffer, cl_uint *size,
                                     const void *host_ptr);                            /* :368 */
void ocl_finish_(bigdft_command_queue *command_queue);                                  /* :374 */
void ocl_enqueue_barrier_(bigdft_command_queue *command_queue);                         /* :377 */
void ocl_clean_command_queue_(bigdft_command_queue *command_queue);                     /* :379 */
void ocl_clean_(bigdft_context *context);                                               /* :381 */
void nanosec_(unsigned long long *t);   /* :306, real-time clock in ns since the epoch */
void init_event_list_(bigdft_context *context);                                         /* :309 */
void print_event_list_(bigdft_context *context);                                        /* :311 */

/* compress / uncompress: OpenCL_wrappers.h:814-905 (Uncompress.c:596-640) */
void uncompress_d_(bigdft_command_queue *command_queue, cl_uint *dimensions, cl_uint *nseg_c, cl_uint *nvctr_c,
                   cl_mem *keyg_c, cl_mem *keyv_c, cl_uint *nseg_f, cl_uint *nvctr_f, cl_mem *keyg_f,
                   cl_mem *keyv_f, cl_mem *psi_c, cl_mem *psi_f, cl_mem *psi_out);          /* :814 */
void compress_d_(bigdft_command_queue *command_queue, cl_uint *dimensions, cl_uint *nseg_c, cl_uint *nvctr_c,
                 cl_mem *keyg_c, cl_mem *keyv_c, cl_uint *nseg_f, cl_uint *nvctr_f, cl_mem *keyg_f,
                 cl_mem *keyv_f, cl_mem *psi_c, cl_mem *psi_f, cl_mem *psi);                /* :833 */
void uncompress_scale_d_(bigdft_command_queue *command_queue, cl_uint *dimensions, cl_double *h, cl_double *c,
                         cl_uint *nseg_c, cl_uint *nvctr_c, cl_mem *keyg_c, cl_mem *keyv_c, cl_uint *nseg_f,
                         cl_uint *nvctr_f, cl_mem *keyg_f, cl_mem *keyv_f, cl_mem *psi_c, cl_mem *psi_f,
                         cl_mem *psi_out);                                                 /* :864 */
void compress_scale_d_(bigdft_command_queue *command_queue, cl_uint *dimensions, cl_double *h, cl_double *c,
                       cl_uint *nseg_c, cl_uint *nvctr_c, cl_mem *keyg_c, cl_mem *keyv_c, cl_uint *nseg_f,
                       cl_uint *nvctr_f, cl_mem *keyg_f, cl_mem *keyv_f, cl_mem *psi_c, cl_mem *psi_f,
                       cl_mem *psi);                                                       /* :885 */
void scale_psi_d_(bigdft_command_queue *command_queue, cl_uint *nvctr_c, cl_uint *nvctr_f, cl_double *h,
                  cl_double *c, cl_mem *psi_c, cl_mem *psi_f);                               /* :846 */

/* 1D rotated passes: OpenCL_wrappers.h:390-512, 619 */
void syn1d_d_(bigdft_command_queue *command_queue, cl_uint *n, cl_uint *ndat, cl_mem *psi, cl_mem *out);      /* :431 */
void syngrow1d_d_(bigdft_command_queue *command_queue, cl_uint *n, cl_uint *ndat, cl_mem *psi, cl_mem *out);  /* :439 */
void ana1d_d_(bigdft_command_queue *command_queue, cl_uint *n, cl_uint *ndat, cl_mem *psi, cl_mem *out);      /* :390 */
void anashrink1d_d_(bigdft_command_queue *command_queue, cl_uint *n, cl_uint *ndat, cl_mem *psi, cl_mem *out); /* :398 */
void magicfilter1d_d_(bigdft_command_queue *command_queue, cl_uint *n, cl_uint *ndat, cl_mem *psi, cl_mem *out); /* :469 */
void magicfiltergrow1d_d_(bigdft_command_queue *command_queue, cl_uint *n, cl_uint *ndat, cl_mem *psi,
                          cl_mem *out);                                                    /* :477 */
void magicfilter1d_t_d_(bigdft_command_queue *command_queue, cl_uint *n, cl_uint *ndat, cl_mem *psi,
                        cl_mem *out);                                                      /* :485 */
void magicfiltershrink1d_d_(bigdft_command_queue *command_queue, cl_uint *n, cl_uint *ndat, cl_mem *psi,
                            cl_mem *out);                                                  /* :493 */
void magicfilter1d_pot_d_(bigdft_command_queue *command_queue, cl_uint *n, cl_uint *ndat, cl_mem *psi,
                          cl_mem *pot, cl_mem *out);                                       /* :512 */
void kinetic1d_d_(bigdft_command_queue *command_queue, cl_uint *n, cl_uint *ndat, cl_double *h, cl_double *c,
                  cl_mem *x, cl_mem *y, cl_mem *workx, cl_mem *worky, cl_double *ekin);    /* :619 */

/* 3D operators: OpenCL_wrappers.h:419-574, 629-639, 1228-1229 */
void syn_self_d_(bigdft_command_queue *command_queue, cl_uint *dimensions, cl_mem *psi, cl_mem *out);        /* :458 */
void ana_self_d_(bigdft_command_queue *command_queue, cl_uint *dimensions, cl_mem *psi, cl_mem *out);        /* :421 */
void syn_self_d_generic_(bigdft_command_queue *command_queue, cl_uint *dimensions, cl_uint *periodic,
                         cl_mem *psi, cl_mem *out);                                        /* :460 */
void ana_self_d_generic_(bigdft_command_queue *command_queue, cl_uint *dimensions, cl_uint *periodic,
                         cl_mem *psi, cl_mem *out);                                        /* :423 */
void syn_d_generic_(bigdft_command_queue *command_queue, cl_uint *dimensions, cl_uint *periodic, cl_mem *tmp,
                    cl_mem *psi, cl_mem *out);                                             /* :456 */
void ana_d_generic_(bigdft_command_queue *command_queue, cl_uint *dimensions, cl_uint *periodic, cl_mem *tmp,
                    cl_mem *psi, cl_mem *out);                                             /* :419 */
void magic_filter_3d_generic_(bigdft_command_queue *command_queue, cl_uint *dimensions, cl_uint *periodic,
                              cl_mem *tmp, cl_mem *tmp_dot, cl_mem *psi, cl_mem *out);     /* :1229 */
void magic_filter_t_3d_generic_(bigdft_command_queue *command_queue, cl_uint *dimensions, cl_uint *periodic,
                                cl_mem *tmp, cl_mem *tmp_dot, cl_mem *psi, cl_mem *out);   /* :1228 */
void potential_application_d_generic_(bigdft_command_queue *command_queue, cl_uint *dimensions,
                                      cl_uint *periodic, cl_mem *tmp, cl_mem *tmp_dot, cl_mem *psi, cl_mem *out,
                                      cl_mem *pot, cl_double *epot);                       /* :574 */
void kinetic_d_generic_(bigdft_command_queue *command_queue, cl_uint *dimensions, cl_uint *periodic,
                        cl_double *h, cl_mem *x, cl_mem *y, cl_mem *work_x, cl_mem *work_y);  /* :639 */
void kinetic_d_(bigdft_command_queue *command_queue, cl_uint *dimensions, cl_double *h, cl_mem *x, cl_mem *y,
                cl_mem *work_x, cl_mem *work_y);                                           /* :629 */
void magicfilter_den_d_generic_(bigdft_command_queue *command_queue, cl_uint *dimensions, cl_uint *periodic,
                                cl_mem *tmp, cl_mem *psi, cl_mem *out);                    /* :542 */

/* BLAS-1 with FP64 reductions: OpenCL_wrappers.h:663-767 */
void dot_d_(bigdft_command_queue *command_queue, cl_uint *n, cl_mem *x, cl_mem *y, cl_mem *work1, cl_mem *work2,
            cl_double *out);                                                              /* :718 */
void dot_d_async_(bigdft_command_queue *command_queue, cl_uint *n, cl_mem *x, cl_mem *y, cl_mem *work1,
                  cl_mem *work2, cl_double *out);                                         /* :728 */
void nrm2sq_d_(bigdft_command_queue *command_queue, cl_uint *n, cl_mem *in, cl_mem *work1, cl_mem *work2,
               cl_double *out);                                                           /* :674 */
void axpy_d_(bigdft_command_queue *command_queue, cl_uint *n, cl_double *alpha, cl_mem *x, cl_mem *y,
             cl_mem *z);                                                                  /* :685 */
void axpy_self_d_(bigdft_command_queue *command_queue, cl_uint *n, cl_double *alpha, cl_mem *x, cl_mem *y); /* :693 */
void scal_d_(bigdft_command_queue *command_queue, cl_uint *n, cl_double *alpha, cl_mem *x, cl_mem *y);      /* :701 */
void scal_self_d_(bigdft_command_queue *command_queue, cl_uint *n, cl_double *alpha, cl_mem *x);            /* :708 */
void copy_d_(bigdft_command_queue *command_queue, cl_uint *n, cl_mem *x, cl_mem *y);                        /* :742 */
void set_d_(bigdft_command_queue *command_queue, cl_uint *n, cl_double *value, cl_mem *x);                  /* :735 */

/* compositions: OpenCL/Hamiltonian.c:41-172, Density.c:37-55, Preconditioner.c:130-360 */
void ocl_fulllocham_generic_(bigdft_command_queue *command_queue, cl_uint *dimensions, cl_uint *periodic,
                             cl_double *h, cl_uint *nseg_c, cl_uint *nvctr_c, cl_mem *keyg_c, cl_mem *keyv_c,
                             cl_uint *nseg_f, cl_uint *nvctr_f, cl_mem *keyg_f, cl_mem *keyv_f, cl_mem *psi_c,
                             cl_mem *psi_f, cl_mem *pot, cl_mem *psi, cl_mem *out, cl_mem *work, cl_mem *kinres,
                             cl_double *epot, cl_double *ekinpot);                          /* Hamiltonian.c:41 */
void ocl_fulllocham_generic_k_(bigdft_command_queue *command_queue, cl_uint *dimensions, cl_uint *periodic,
                               cl_double *h, cl_double *k, cl_uint *nseg_c, cl_uint *nvctr_c, cl_mem *keyg_c,
                               cl_mem *keyv_c, cl_uint *nseg_f, cl_uint *nvctr_f, cl_mem *keyg_f, cl_mem *keyv_f,
                               cl_mem *psi_c_r, cl_mem *psi_f_r, cl_mem *psi_c_i, cl_mem *psi_f_i, cl_mem *pot,
                               cl_mem *psi_r, cl_mem *out_r, cl_mem *work_r, cl_mem *psi_i, cl_mem *out_i,
                               cl_mem *work_i, cl_mem *kinres_r, cl_mem *kinres_i, cl_uint *nspinor,
                               cl_double *epot, cl_double *ekinpot);                        /* Hamiltonian.c:105 */
void ocl_daub_to_isf_(bigdft_command_queue *command_queue, cl_uint *dimensions, cl_uint *periodic,
                      cl_uint *nseg_c, cl_uint *nvctr_c, cl_mem *keyg_c, cl_mem *keyv_c, cl_uint *nseg_f,
                      cl_uint *nvctr_f, cl_mem *keyg_f, cl_mem *keyv_f, cl_mem *psi_c, cl_mem *psi_f,
                      cl_mem *psi, cl_mem *out, cl_mem *work, cl_mem *kinres);              /* Hamiltonian.c:89 */
void ocl_isf_to_daub_(bigdft_command_queue *command_queue, cl_uint *dimensions, cl_uint *periodic,
                      cl_uint *nseg_c, cl_uint *nvctr_c, cl_mem *keyg_c, cl_mem *keyv_c, cl_uint *nseg_f,
                      cl_uint *nvctr_f, cl_mem *keyg_f, cl_mem *keyv_f, cl_mem *psi_c, cl_mem *psi_f,
                      cl_mem *psi, cl_mem *out, cl_mem *work, cl_mem *kinres);              /* Hamiltonian.c:74 */
void ocl_locden_generic_(bigdft_command_queue *command_queue, cl_uint *dimensions, cl_uint *periodic,
                         cl_double *hfac, cl_uint *nseg_c, cl_uint *nvctr_c, cl_mem *keyg_c, cl_mem *keyv_c,
                         cl_uint *nseg_f, cl_uint *nvctr_f, cl_mem *keyg_f, cl_mem *keyv_f, cl_mem *psi_c,
                         cl_mem *psi_f, cl_mem *psi, cl_mem *out, cl_mem *work, cl_mem *pot); /* Density.c:37 */
void ocl_preconditioner_generic_(bigdft_command_queue *command_queue, cl_uint *dimensions, cl_uint *periodic,
                                 cl_double *h, cl_double *c, cl_uint *ncong, cl_uint *nseg_c, cl_uint *nvctr_c,
                                 cl_mem *keyg_c, cl_mem *keyv_c, cl_uint *nseg_f, cl_uint *nvctr_f,
                                 cl_mem *keyg_f, cl_mem *keyv_f, cl_mem *psi_c, cl_mem *psi_f, cl_mem *psi_c_r,
                                 cl_mem *psi_f_r, cl_mem *psi_c_b, cl_mem *psi_f_b, cl_mem *psi_c_d,
                                 cl_mem *psi_f_d, cl_mem *work1, cl_mem *work2, cl_mem *work3,
                                 cl_mem *work4);                                           /* Preconditioner.c:130 */
void ocl_preconditioner_generic_k_(bigdft_command_queue *command_queue, cl_uint *dimensions, cl_uint *periodic,
                                   cl_double *h, cl_double *k, cl_double *c, cl_uint *ncong, cl_uint *nseg_c,
                                   cl_uint *nvctr_c, cl_mem *keyg_c, cl_mem *keyv_c, cl_uint *nseg_f,
                                   cl_uint *nvctr_f, cl_mem *keyg_f, cl_mem *keyv_f, cl_mem *psi_c_r,
                                   cl_mem *psi_f_r, cl_mem *psi_c_i, cl_mem *psi_f_i, cl_mem *psi_c_r_r,
                                   cl_mem *psi_f_r_r, cl_mem *psi_c_r_i, cl_mem *psi_f_r_i, cl_mem *psi_c_b_r,
                                   cl_mem *psi_f_b_r, cl_mem *psi_c_b_i, cl_mem *psi_f_b_i, cl_mem *psi_c_d_r,
                                   cl_mem *psi_f_d_r, cl_mem *psi_c_d_i, cl_mem *psi_f_d_i, cl_mem *work1_r,
                                   cl_mem *work2_r, cl_mem *work3_r, cl_mem *work4_r, cl_mem *work1_i,
                                   cl_mem *work2_i, cl_mem *work3_i, cl_mem *work4_i, cl_uint *nspinor,
                                   cl_double *norm_sq_cf);                                 /* Preconditioner.c:247 */

/* last error recorded by any entry point of the process, then reset to 0
 * (no counterpart in the reference, which exits on error) */
int wvlh_get_last_error(void);
const char *wvlh_error_string(int code);
/* device pointer of a buffer handle (for interoperability and tests) */
void *wvlh_mem_ptr(cl_mem mem);

/* --------------------------------------------------------------------- */
/* 2. batched ABI (new)                                                   */
/* --------------------------------------------------------------------- */
typedef struct wvlh_ctx wvlh_ctx;
typedef struct wvlh_batch wvlh_batch;

/* One localisation region: coarse cells per dimension (n1+1, n2+1, n3+1),
 * periodicity, coarse grid spacing and the reference's 1-based keys (HOST
 * arrays, keyg(2,nseg) / keyv(nseg), wavelib compression.f90:29-39). */
typedef struct {
    int n[3];
    int periodic[3];
    double hgrid[3];
    int nseg_c, nseg_f;
    const int32_t *keyg_c, *keyv_c;
    const int32_t *keyg_f, *keyv_f;
} wvlh_locreg;

int wvlh_ctx_create(int device, wvlh_ctx **ctx);
int wvlh_ctx_destroy(wvlh_ctx *ctx);
/* stream (cudaStream_t) all calls of this context are issued on; 0 = legacy */
int wvlh_ctx_set_stream(wvlh_ctx *ctx, void *stream);
int wvlh_ctx_synchronize(wvlh_ctx *ctx);

/* Validate and upload the keys of nlr regions and lay out norb orbitals:
 * orbital o lives in region orb_lr[o]; its coefficients [psi_c | psi_f]
 * start at wvlh_batch_psi_offset(o) (orbitals packed in order); its local
 * potential / density grid (ISF points, x fastest) starts at element
 * pot_offset[o] of the pot/rho arrays (NULL: all orbitals at offset 0). */
int wvlh_batch_create(wvlh_ctx *ctx, int nlr, const wvlh_locreg *lrs, int norb, const int32_t *orb_lr,
                      const int64_t *pot_offset, wvlh_batch **batch);
int wvlh_batch_destroy(wvlh_batch *batch);
int64_t wvlh_batch_psi_size(const wvlh_batch *batch);    /* total coefficient count */
int64_t wvlh_batch_psi_offset(const wvlh_batch *batch, int orb);
int64_t wvlh_batch_scratch_bytes(const wvlh_batch *batch, int precision);

/* Resident regions and per-launch orbital batches (serving: many independent
 * clients, each with its own box, buffers and density; no counterpart in the
 * reference, whose host owns one set of buffers per process).
 *
 * A region is one client's localisation region with its keys validated,
 * decoded and uploaded once; it must outlive the batches that use it. */
typedef struct wvlh_region wvlh_region;
int wvlh_region_create(wvlh_ctx *ctx, const wvlh_locreg *lr, wvlh_region **region);
int wvlh_region_destroy(wvlh_region *region);
int64_t wvlh_region_psi_size(const wvlh_region *region);   /* nvctr_c + 7 nvctr_f */
int64_t wvlh_region_grid_size(const wvlh_region *region);  /* ISF (potential / density) points */
int64_t wvlh_region_scratch_bytes(const wvlh_region *region, int precision);  /* per orbital */

/* One orbital of an orbital batch: its region and its own DEVICE buffers
 * (precision of the launch): psi [psi_c | psi_f], hpsi and the region's ISF
 * potential for wvlh_locham_batched; rho (FP64 ISF grid, accumulated) for
 * wvlh_locden_batched.  Unused buffers may be NULL. */
typedef struct {
    const wvlh_region *region;
    const void *psi;
    void *hpsi;
    const void *pot;
    double *rho;
} wvlh_orbital;
/* Build a batch over orbitals of any regions.  Its tables go to a grow-only
 * arena of the context, written by a copy queued on the context's stream, so
 * that a new batch costs no device allocation once the arena is large enough;
 * launches of a batch must be queued before the next orbital batch of the
 * same context is created (later launches return WVLH_ERR_STALE).  Launch
 * with NULL psi/pot/hpsi (locham) or psi/rho (locden): each orbital's own
 * buffers are used.  Orbitals that share rho must share their region. */
int wvlh_batch_create_orbitals(wvlh_ctx *ctx, int norb, const wvlh_orbital *orbs, wvlh_batch **batch);

/* Hpsi for all orbitals of the batch.  precision 32: psi/pot/hpsi are float,
 * 64: double.  Device pointers.  ekin/epot: device arrays of norb doubles
 * (<psi|T|psi> and <psi|V|psi> per orbital, the reference's per-orbital ekin
 * and epot of local_hamiltonian_ket).  accumulate != 0 adds into hpsi like
 * compress_and_accumulate_mixed; 0 overwrites like compress_d. */
int wvlh_locham_batched(wvlh_batch *batch, int precision, const void *psi, const void *pot, void *hpsi,
                        double *ekin, double *epot, int accumulate);
/* same with HOST buffers (pinned for full speed): copies in, computes, copies
 * out, synchronises.  Batches of 16 orbitals or more go through in chunks of
 * consecutive orbitals (8 or more each, up to 32 chunks): all uploads queue
 * back to back on one stream of the context, each chunk's kernels run on the
 * context's stream once its input has arrived, and each chunk's download
 * queues on a third stream once it is computed, so both copy directions and
 * the kernels overlap. */
int wvlh_locham_batched_host(wvlh_batch *batch, int precision, const void *psi, const void *pot, void *hpsi,
                             double *ekin, double *epot);
/* Density of all orbitals: rho[pot_offset[o] + r] += hfac[o] * |psi_o(r)|^2 on
 * the ISF grid (local_partial_density, sumrho.f90:377-577; ocl_locden_generic,
 * OpenCL/Density.c:37).  hfac: device array of norb doubles (kwgt*occ/vol);
 * rho: device FP64, accumulated.  Orbitals sharing a density offset must share
 * their region.  Fixed summation order: deterministic. */
int wvlh_locden_batched(wvlh_batch *batch, int precision, const void *psi, const double *hfac, double *rho);
/* Preconditioner of all orbitals: ncong CG iterations on
 * D^-1/2 A (c_o + T) S D^-1/2 x = rhs, then x *= D^-1/2, per orbital, exactly the
 * recurrence of ocl_preconditioner_generic (OpenCL/Preconditioner.c:130-195)
 * with the shifts c_o = cprec[o] (device, norb doubles).  x (in: initial guess,
 * out: result) and rhs are device arrays in the batch layout; hist (optional,
 * device, (ncong+1)*norb doubles) receives the squared residual norms, entry 0
 * the initial one.  Scalars stay on the device: no host synchronisation. */
int wvlh_precond_batched(wvlh_batch *batch, int precision, int ncong, const double *cprec, void *x, const void *rhs,
                         double *hist);
/* Overlap S = Psi^T Psi (norb x norb, FP64, full symmetric, row-major) of
 * norb coefficient rows of length K at row stride ld (device; precision 32:
 * float rows widened to FP64, 64: double) on FP64 tensor cores; the
 * reference's getOverlap syrk (wfn_opt/orthogonality.f90:2675) summed in a
 * fixed order. */
int wvlh_overlap(wvlh_ctx *ctx, int precision, int norb, int64_t K, int64_t ld, const void *psi, double *S);
/* Subspace matrix L[i][j] = <psi_i | hpsi_j> (norb x norb, FP64, row-major:
 * row i, column j) of two panels with the same layout: the Lagrange
 * multipliers of orthoconstraint (wfn_opt/orthogonality.f90:375-625,
 * subspace_matrix :196-224, gemm('T','N')), on the same FP64 tensor-core
 * kernel, every tile of the square, splits summed in a fixed order. */
int wvlh_subspace_matrix(wvlh_ctx *ctx, int precision, int norb, int64_t K, int64_t ld, const void *psi,
                         const void *hpsi, double *L);
/* Panel apply out = beta out + alpha M psi (FP64, device): M is norb x norb
 * row-major (lower != 0: lower triangular, the slices above the diagonal are
 * skipped), psi and out are norb rows of K values at row stride ld (out
 * must not alias psi).  The psi-sized
 * products of the orthonormalisation (wfn_opt/orthogonality.f90): Cholesky
 * psi <- L^-1 psi (dtrtri then dtrmm, :2351-2366), Loewdin psi <- S^-1/2 psi
 * (:2486), and the Lagrange step hpsi <- hpsi - L^T psi (subspace_update,
 * :254-271; M = L^T, alpha = -1, beta = 1), on FP64 tensor cores, the
 * contraction in a fixed order. */
int wvlh_panel_apply(wvlh_ctx *ctx, int norb, int64_t K, int64_t ld, const double *M, int lower, double alpha,
                     const double *psi, double beta, double *out);
/* Compressed scalar products out[i*nb + j] = <a_i|b_j> (FP64) between na
 * vectors on the keys of region ra (row stride lda) and nb vectors on the
 * keys of region rb (row stride ldb), both regions with the same box (keys
 * are linear indices of one grid): the reference's wpdot
 * (wavelib/scalprod.f90:3222), coarse and 7 fine components, with its
 * pairing of segments — each b segment takes its overlap with the first a
 * segment it meets (the whole common part whenever each b segment meets at
 * most one a segment, as for projectors inside a wavefunction's region).
 * precision 32: float vectors, FP64 sums; 64: double.  Device pointers. */
int wvlh_wpdot(wvlh_ctx *ctx, int precision, const wvlh_region *ra, int na, const void *a, int64_t lda,
               const wvlh_region *rb, int nb, const void *b, int64_t ldb, double *out);
/* Nonlocal pseudopotential projectors (NonLocalHamiltonianApplication,
 * hpsiortho.f90:1044-1125, through DFT_PSP_projectors_iter_apply,
 * modules/psp_projectors.f90:585-712): for every orbital psi on the keys of
 * psi_region and every atom a, with p_1..p_m the atom's m = nproj[a]
 * projectors on the keys of proj_regions[a] (same box as psi_region) and h its
 * m x m coefficient matrix,
 *     c_i = <p_i|psi>  (pr_dot_psi, locregs/compression.f90:505),
 *     hc  = h c        (apply_hij_coeff, orbitals/pseudopotentials.f90:1208),
 *     eproj += c . hc  (cproj_dot, compression.f90:540),
 *     hpsi += sum_i hc_i p_i on the common points (cproj_pr_p_psi, :562).
 * The common points are the reference's masks between the wavefunction's and
 * the projector's segments (count_wblas_segs / fill_wblas_segs,
 * locregs/scalar_product.f90:1012-1187: each projector segment meets the first
 * wavefunction segment it overlaps), coarse and 7 fine components.  Atoms are
 * applied in order, each orbital's sums in a fixed order (deterministic).
 * proj: DEVICE doubles, per atom its m vectors of wvlh_region_psi_size(
 * proj_regions[a]) values one after another, atoms one after another; copied
 * at creation.  hij: HOST doubles, per atom m x m row-major, atoms one after
 * another; copied.  m <= 32 per atom.  Regions must outlive the object. */
typedef struct wvlh_nlpsp wvlh_nlpsp;
int wvlh_nlpsp_create(wvlh_ctx *ctx, const wvlh_region *psi_region, int natoms, const wvlh_region *const *proj_regions,
                      const int *nproj, const double *proj, const double *hij, wvlh_nlpsp **nl);
/* norb orbitals on psi_region (row stride ld >= its psi size), DEVICE FP64:
 * hpsi += V_nl psi, eproj[o] = sum over atoms of c . hc (written). */
int wvlh_nlpsp_apply(wvlh_nlpsp *nl, int norb, const double *psi, int64_t ld, double *hpsi, double *eproj);
int wvlh_nlpsp_destroy(wvlh_nlpsp *nl);
/* Hartree potential of a density on a periodic real-space (ISF) grid, the
 * reference's PSolver for periodic boundary conditions (Periodic_Kernel and
 * fourtrans_isf, psolver/src/Build_Kernel.f90:16-262; P_multkernel_NO,
 * PSolver_Base_new.f90:2515-2640; scal 1/(n1 n2 n3), createKernel.f90:299):
 * V^(k) = rho^(k) phi^_x phi^_y phi^_z / (pi g^2) with the order-16 ISF
 * Fourier factors, the k = 0 term set to offset / h^3.  n: grid points per
 * dimension (x fastest; even, >= 16), h: spacings (bohr), rho/pot: DEVICE FP64
 * arrays of n1 n2 n3 values (pot may be rho when eh is NULL).  eh (DEVICE, one
 * double, or NULL): the Hartree energy 0.5 sum(rho V) h1 h2 h3
 * (PSolver_Main.f90:403).  FFTs by cuFFT, plans kept per context and grid. */
int wvlh_psolver_periodic(wvlh_ctx *ctx, const int n[3], const double h[3], const double *rho, double *pot,
                          double offset, double *eh);
/* Hartree potential with free (isolated) boundary conditions, the reference's
 * PSolver for geocode 'F' (Free_Kernel, psolver/src/Build_Kernel.f90:985-1175,
 * from the 89-Gaussian expansion of 1/r, gequad :1679-1873, and the order-16
 * ISF; scal h1 h2 h3 / (N1 N2 N3), createKernel.f90:439): rho zero-padded to
 * at least twice each dimension, multiplied by the kernel's Fourier table,
 * the first octant kept.  n: points per dimension (x fastest, 2..4096), h:
 * spacings (bohr), rho/pot: DEVICE FP64 (pot may be rho when eh is NULL).
 * eh (DEVICE, or NULL): 0.5 sum(rho V) h1 h2 h3.  The kernel table, FFT plans
 * and padded buffers are built at the first call for a grid and kept. */
int wvlh_psolver_free(wvlh_ctx *ctx, const int n[3], const double h[3], const double *rho, double *pot, double *eh);
/* Host only (no device work): the padded FFT lengths nf and the free kernel's
 * 1D tables that wvlh_psolver_free sums on the device: per Gaussian g = 0..88
 * a row [C_x(0..N1/2) | C_y(0..N2/2) | C_z(0..N3/2)], then the 89 weights;
 * K(k3, k2, k1) = sum_g C_x(k1) (C_z(k3) (C_y(k2) w_g)), g from 88 down to 0.
 * With tab NULL returns the number of doubles; otherwise fills tab (cap
 * doubles) and returns that number; on an error, minus the error code. */
int64_t wvlh_psolver_free_tables(const int n[3], const double h[3], int nf[3], double *tab, int64_t cap);
/* Hartree potential with surface boundary conditions (x and z periodic, y
 * free: the reference's PSolver for geocode 'S', Surfaces_Kernel,
 * psolver/src/Build_Kernel.f90:279-864; scal -4 pi h_y / N, createKernel.f90:
 * 374): for each in-plane frequency the 1D Green's function along y of the
 * order-16 ISF (exp(-mu |y|) / mu, |y| at zero frequency), rho zero-padded
 * along y to at least twice n2.  Arguments and results as wvlh_psolver_free;
 * the kernel table (built once per grid on the host's threads), FFT plans and
 * padded buffers are kept by the context. */
int wvlh_psolver_surface(wvlh_ctx *ctx, const int n[3], const double h[3], const double *rho, double *pot,
                         double *eh);
/* Host only (no device work): the padded y length N2 and the surface kernel
 * table K(k3, ky, k1), (n3/2+1, N2/2+1, n1/2+1) doubles, that
 * wvlh_psolver_surface multiplies by.  With tab NULL returns the number of
 * doubles; otherwise fills tab (cap doubles) and returns that number; on an
 * error, minus the error code. */
int64_t wvlh_psolver_surface_table(const int n[3], const double h[3], int *N2, double *tab, int64_t cap);
/* Hartree potential with wire boundary conditions (z periodic, x and y
 * free: the reference's PSolver for geocode 'W', Wires_Kernel,
 * psolver/src/Build_Kernel.f90:2244-2364, from the Gaussian fits of log r
 * and K0(r) in gaussfit_wires.inc; scal -2 h_x h_y / N, createKernel.f90:
 * 502): rho zero-padded in x and y to at least twice each.  Arguments and
 * results as wvlh_psolver_free; the kernel table (built once per grid on the
 * host's threads), FFT plans and padded buffers are kept by the context. */
int wvlh_psolver_wire(wvlh_ctx *ctx, const int n[3], const double h[3], const double *rho, double *pot, double *eh);
/* Host only (no device work): the padded x and y lengths nf and the wire
 * kernel table K(kz, ky, kx), (n3/2+1, nf[1]/2+1, nf[0]/2+1) doubles.  With
 * tab NULL returns the number of doubles; otherwise fills tab (cap doubles)
 * and returns that number; on an error, minus the error code. */
int64_t wvlh_psolver_wire_table(const int n[3], const double h[3], int nf[2], double *tab, int64_t cap);
/* Exchange-correlation potential of the reference's default functional
 * (ixc = 1: the Goedecker-Teter-Hutter Pade LDA, ABINIT's xcspol,
 * libABINIT/src/abi_xc_lowlevel/abi_xcspol.F90:105-250), spin-unpolarised,
 * for npts points of the total density rho (DEVICE FP64, positive: the
 * reference keeps it >= 1e-20): vxc[i] = v_xc(rho[i]), or vxc[i] += v_xc when
 * accumulate (vxc may be rho).  energies (DEVICE double[2], or NULL):
 * exc = dvol sum eps_xc rho, evxc = dvol sum v_xc rho (xc_energy_new,
 * bigdft/src/orbitals/xc.f90:763-925).  Replaces XC_potential
 * (xcPSolver/xcenergy.f90:428) for ixc = 1, nspin = 1, no core density. */
int wvlh_xc_lda(wvlh_ctx *ctx, int64_t npts, const double *rho, double *vxc, int accumulate, double dvol,
                double *energies);
/* The Kohn-Sham potential of a periodic box from the total density (the
 * reference's updatePotential, bigdft/src/modules/rhopotential.f90:29-125,
 * nspin = 1, ixc = 1): pot = (V_H[rho] + vext) + V_xc[rho], V_H as
 * wvlh_psolver_periodic with offset 0; vext may be NULL.  pot must not alias
 * rho or vext.  energies (DEVICE double[3], or NULL): eh = 0.5 dvol sum rho
 * V_H, exc, evxc.  One pass after the inverse FFT forms the sum and the three
 * energies. */
int wvlh_ks_potential_periodic(wvlh_ctx *ctx, const int n[3], const double h[3], const double *rho,
                               const double *vext, double *pot, double *energies);
/* The same Kohn-Sham potential with free boundary conditions (V_H as
 * wvlh_psolver_free). */
int wvlh_ks_potential_free(wvlh_ctx *ctx, const int n[3], const double h[3], const double *rho, const double *vext,
                           double *pot, double *energies);
/* Spin-polarised LDA (ixc = 1, nspin = 2: xcspol's spin interpolation with the
 * fit's ferromagnetic differences, abi_xcspol.F90:113-116, 355-395) for npts
 * points of the spin densities (DEVICE FP64): vxc_up/dn[i] = v_xc,sigma (or
 * added when accumulate; vxc_up may be rho_up, vxc_dn rho_dn).  energies
 * (DEVICE double[2], or NULL): exc = dvol sum eps (up + dn), evxc = dvol
 * sum_sigma v_sigma rho_sigma. */
int wvlh_xc_lsda(wvlh_ctx *ctx, int64_t npts, const double *rho_up, const double *rho_dn, double *vxc_up,
                 double *vxc_dn, int accumulate, double dvol, double *energies);
/* The Kohn-Sham potential of updatePotential for any of the reference's
 * boundary conditions, bc = 0 periodic (offset 0), 1 free, 2 surface, 3 wire:
 * pot = (V_H[rho] + vext) + V_xc[rho], V_H as wvlh_psolver_periodic / _free /
 * _surface / _wire; arguments, aliasing rules and energies as
 * wvlh_ks_potential_periodic.  rhocore (DEVICE, or NULL): a core density for
 * the nonlinear core correction, added to rho for V_xc and E_xc only, with
 * evxc counting the valence density alone (XC_potential with rhocore,
 * xcPSolver/xcenergy.f90:720-725, substract_from_vexcu :850-882). */
int wvlh_ks_potential_bc(wvlh_ctx *ctx, int bc, const int n[3], const double h[3], const double *rho,
                         const double *rhocore, const double *vext, double *pot, double *energies);
/* The Kohn-Sham potentials of updatePotential with nspin = 2
 * (rhopotential.f90:87-120): V_H of the total density (free_bc: the
 * boundary-condition code of wvlh_ks_potential_bc; 0 periodic, 1 free,
 * 2 surface, 3 wire), pot_sigma = (V_H + vext) + V_xc,sigma;
 * energies as wvlh_ks_potential_periodic (evxc summed over both spins);
 * rhocore as wvlh_ks_potential_bc, half of it on each spin.
 * pot_up and pot_dn are distinct and alias no input. */
int wvlh_ks_potential_spin(wvlh_ctx *ctx, int free_bc, const int n[3], const double h[3], const double *rho_up,
                           const double *rho_dn, const double *rhocore, const double *vext, double *pot_up,
                           double *pot_dn, double *energies);
/* Measured block size of the plane kernels: times reps calls of
 * wvlh_locham_batched (after one warm-up each) with every block size the
 * kernels are compiled for (FP32 1024/512/384/256/128, FP64 512/384/256/128),
 * keeps the fastest in the batch and in a process-wide table keyed by the
 * batch's shape (precision and every orbital's box), which batches of the
 * same shape created later start from.  Arguments as wvlh_locham_batched
 * (hpsi, ekin, epot are overwritten); chosen: the pick; cand/ms (up to 5
 * entries each, or NULL): the candidates and their ms per call; ncand: how
 * many were timed. */
int wvlh_batch_autotune(wvlh_batch *batch, int precision, const void *psi, const void *pot, void *hpsi,
                        double *ekin, double *epot, int reps, int *chosen, int *cand, double *ms, int *ncand);
/* The same measured choice for the preconditioner operator of
 * wvlh_precond_batched (ncong CG iterations per timed call on the caller's
 * x and rhs; x is overwritten), kept apart from the local Hamiltonian's: the
 * preconditioner's plane kernels run fewer passes per plane.  Packed batches
 * only, as wvlh_precond_batched. */
int wvlh_batch_autotune_precond(wvlh_batch *batch, int precision, int ncong, const double *cprec, void *x,
                                const void *rhs, int reps, int *chosen, int *cand, double *ms, int *ncand);
/* The block sizes the batch launches with: {plane kernels FP32, FP64, z kernel
 * FP32, FP64} of the local Hamiltonian (its plane sizes serve the density as
 * well), then the same four of the preconditioner.  The autotuners above also time the FP32 z kernel's
 * sizes (256, 320, 384) after the plane kernels' pick. */
int wvlh_batch_block_sizes(const wvlh_batch *batch, int *sizes8);
/* FP64, one kernel per 1D pass (the OpenCL backend's structure) */
int wvlh_locham_plain_batched(wvlh_batch *batch, const double *psi, const double *pot, double *hpsi,
                              double *ekin, double *epot);

/* CUDA graph of one wvlh_locham_batched call with fixed arguments (a packed
 * batch applied at every SCF iteration): the memsets and kernels are captured
 * once (on a private stream) and replayed by wvlh_graph_launch on the
 * context's stream with one launch.  The graph owns its scratch; the batch and
 * the buffers named at capture must outlive it.  Orbital batches are refused
 * (WVLH_ERR_UNSUPPORTED): their tables are replaced by the next batch. */
typedef struct wvlh_graph wvlh_graph;
int wvlh_locham_graph_create(wvlh_batch *batch, int precision, const void *psi, const void *pot, void *hpsi,
                             double *ekin, double *epot, int accumulate, wvlh_graph **graph);
int wvlh_graph_launch(wvlh_graph *graph);
int wvlh_graph_destroy(wvlh_graph *graph);

/* Optional per-kernel timing with CUDA events recorded on the context's
 * stream around the fused kernels (K1 plane-forward, K2 z-pencil, K3
 * plane-backward, energy reduction).  While on, each wvlh_locham_batched call
 * waits for its own events; times accumulate until re-enabled. */
int wvlh_ctx_enable_timing(wvlh_ctx *ctx, int on);
int wvlh_ctx_kernel_times(wvlh_ctx *ctx, double *ms4, long long *ncalls);
/* FMA-pipe throughput of this GPU (TFLOP/s) from a register-resident FMA
 * chain kernel, the compute roof of the fused stencils (precision 32 or 64). */
int wvlh_measure_fma_peak(int precision, int iters, double *tflops);

/* Local Hamiltonian of ONE orbital that allocates nothing.  No counterpart in
 * the reference.  For callers that cannot call cudaMalloc (an application
 * whose memory manager owns every device allocation, a layer that must not
 * grow the device footprint on its own): all tables and scratch of the fused
 * kernels live in a static device array of wvlh_noalloc_capacity() bytes
 * (64 MiB), held on each GPU where this entry point has been used until the
 * process exits.  psi/pot/hpsi/ekin/epot are the caller's DEVICE buffers
 * (precision 32: float, 64: double; ekin/epot one double each); the keys are
 * HOST arrays, 1-based as in the reference, read by copies queued on `stream`
 * (keep them unchanged until the stream reaches the call).  Boxes whose
 * scratch exceeds the capacity return WVLH_ERR_TOO_LARGE.  The first call on
 * a device looks up the device address of the static array (set-up) and keeps
 * it for the life of the process, so resetting the device while the library
 * is loaded is not supported: make that first call before any stream capture.
 * Every call uses the same array,
 * so calls that overlap on the GPU (other streams, other host threads) race:
 * serialise them. */
int wvlh_locham_noalloc(int precision, const int n[3], const int periodic[3], const double hgrid[3], int nseg_c,
                        const int32_t *keyg_c, const int32_t *keyv_c, int nseg_f, const int32_t *keyg_f,
                        const int32_t *keyv_f, const void *psi, const void *pot, void *hpsi, double *ekin,
                        double *epot, void *stream);
size_t wvlh_noalloc_capacity(void);

/* pinned host memory helpers */
void *wvlh_host_alloc(size_t bytes);
void wvlh_host_free(void *p);

#ifdef __cplusplus
}
#endif
#endif
