/*
 * shtns_cuda.h -- device-pointer transforms of shtns_b200, a drop-in for the
 * SHTns 3.5.2 header of the same name (reference shtns_cuda.h:408-442).
 *
 * As in the reference, these transforms work on data already resident in GPU
 * memory, are asynchronous on the plan's compute stream (stream 0 unless set
 * by cushtns_set_streams or cushtns_clone) and a plan must not be used by two
 * host threads at once; clone it per thread or per stream.  Unlike the
 * reference, spat_to_SH-type device transforms never overwrite their spatial
 * input, and any even nlat is accepted (the reference requires a multiple of
 * 64).  The spatial layout is the one requested at shtns_set_grid
 * (theta-contiguous by default, phi-contiguous on request).
 */
#ifndef SHTNS_B200_SHTNS_CUDA_H
#define SHTNS_B200_SHTNS_CUDA_H

#include <cuda_runtime.h>
#include "shtns.h"

#ifdef __cplusplus
extern "C" {
#endif

void cu_spat_to_SH(shtns_cfg shtns, double *Vr, cplx *Qlm, int ltr);                        /* shtns_cuda.h:408 */
void cu_spat_to_SH_float(shtns_cfg shtns, float *Vr, cplx_f *Qlm, int ltr);                 /* shtns_cuda.h:410 */
void cu_SH_to_spat(shtns_cfg shtns, cplx *Qlm, double *Vr, int ltr);                        /* shtns_cuda.h:412 */
void cu_SH_to_spat_float(shtns_cfg shtns, cplx_f *Qlm, float *Vr, int ltr);                 /* shtns_cuda.h:414 */
void cu_spat_to_SHsphtor(shtns_cfg, double *Vt, double *Vp, cplx *Slm, cplx *Tlm, int ltr); /* shtns_cuda.h:416 */
void cu_SHsphtor_to_spat(shtns_cfg, cplx *Slm, cplx *Tlm, double *Vt, double *Vp, int ltr); /* shtns_cuda.h:418 */
void cu_spat_to_SHqst(shtns_cfg, double *Vr, double *Vt, double *Vp, cplx *Qlm, cplx *Slm, cplx *Tlm, int ltr);  /* shtns_cuda.h:420 */
void cu_SHqst_to_spat(shtns_cfg, cplx *Qlm, cplx *Slm, cplx *Tlm, double *Vr, double *Vt, double *Vp, int ltr);  /* shtns_cuda.h:422 */

shtns_cfg cushtns_clone(shtns_cfg shtns, cudaStream_t compute_stream, cudaStream_t transfer_stream);  /* shtns_cuda.h:433 */
int cushtns_init_gpu(shtns_cfg shtns);                                                      /* shtns_cuda.h:439 */
void cushtns_set_streams(shtns_cfg shtns, cudaStream_t compute_stream, cudaStream_t transfer_stream);  /* shtns_cuda.h:442 */

#ifdef __cplusplus
}
#endif

#endif /* SHTNS_B200_SHTNS_CUDA_H */
