/*
 * shtns_b200.h -- entry points of shtns_b200 that have no counterpart in
 * SHTns 3.5.2.  They sit beside the drop-in API of shtns.h / shtns_cuda.h.
 */
#ifndef SHTNS_B200_EXT_H
#define SHTNS_B200_EXT_H

#include <stddef.h>
#include "shtns.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Batched transforms.  After shtns_set_batch(cfg, howmany, spec_dist,
 * spat_dist) every transform of this plan (host and cu_* forms) processes
 * `howmany` independent fields: field i of each spectral array starts at
 * element i*spec_dist (complex elements, >= nlm) and field i of each spatial
 * array at element i*spat_dist (doubles, >= nspat).  howmany = 1 restores the
 * single-field behaviour.  Returns 0, or -1 for invalid arguments.
 * No counterpart in SHTns 3.5.2 (its transforms take one field per call). */
int shtns_set_batch(shtns_cfg, int howmany, long spec_dist, long spat_dist);

/* Error handling.  By default, like SHTns 3.5.2 (sht_init.c:67-72), an invalid
 * plan request prints a message and exits the process.  With
 * shtns_b200_error_mode(1) the failing call instead returns NULL / -1 and the
 * message is kept for shtns_b200_last_error().  Transform errors (invalid
 * sizes, CUDA launch failures) never exit: they are recorded here and the
 * transform returns without writing its outputs. */
void shtns_b200_error_mode(int return_errors);
const char* shtns_b200_last_error(void);
/* 0 if no transform error happened since the last call, else a nonzero code
 * (1 = invalid argument, 2 = CUDA error, 3 = allocation failure);
 * the status is cleared by this call. */
int shtns_b200_status(void);

/* Device used by a plan and bytes of GPU memory it holds: its tables (for a
 * clone, none: they belong to the base plan), including the FP64 and INT8
 * Legendre tables once built, and its work buffers. */
int shtns_b200_device(shtns_cfg);
size_t shtns_b200_device_bytes(shtns_cfg);

/* Number of kernel launches issued by this library since process start (all
 * plans).  Used to count the launches inside a timed region. */
long shtns_b200_launch_count(void);

/* Per-stage GPU timing.  With shtns_b200_set_timing(cfg, 1) every transform
 * records CUDA events around its kernels on the plan's compute stream (one
 * event pair per stage, no host synchronisation).  shtns_b200_stage_times()
 * waits for the recorded events, writes the accumulated milliseconds and call
 * counts of the 6 stages (0 coefficient prologue, 1 Legendre synthesis,
 * 2 FFT synthesis, 3 FFT analysis, 4 Legendre analysis, 5 coefficient
 * epilogue) into ms[6] and calls[6] (either may be NULL), and resets them. */
void shtns_b200_set_timing(shtns_cfg, int on);
int shtns_b200_stage_times(shtns_cfg, double* ms, long* calls);

/* First north-hemisphere latitude row kept by the polar threshold for each
 * order im = 0..mmax (rows closer to the pole are treated as zero, as the
 * reference's PolarOptimize does).  Writes mmax+1 ints; returns mmax+1. */
int shtns_b200_polar_rows(shtns_cfg, int* tm);

/* Exact adjoints (transposes, real inner products with complex numbers
 * taken as pairs of reals) of the scalar device transforms, used for
 * reverse-mode differentiation.  cu_SH_to_spat_adjoint maps a spatial
 * gradient Vg (nspat doubles per field) to the spectral gradient Qg:
 *   Qg_lm = (2 - delta_m0) nphi sum_theta P_lm(theta) G_m(theta),
 *   G_m = (1/nphi) sum_phi Vg e^{-i m phi}  (a quadrature-weight-free analysis);
 * cu_spat_to_SH_adjoint maps a spectral gradient Qg to the spatial gradient
 * Vg (a synthesis with the quadrature weight of each latitude).  Batched by
 * shtns_set_batch like the other transforms; ltr as in cu_SH_to_spat.
 * No counterpart in SHTns 3.5.2. */
void cu_SH_to_spat_adjoint(shtns_cfg, double *Vg, cplx *Qg, int ltr);
void cu_spat_to_SH_adjoint(shtns_cfg, cplx *Qg, double *Vg, int ltr);

/* Tuning options of a plan.  option 1: latitude pairs per FFT CTA (1, 2, 4,
 * 8 where the fused chain's buffer fits; 0 = automatic); option 2: recurrence checkpoint spacing (8, 16, 32; rebuilds
 * the checkpoint table; not for clones or plans that have clones); option 3:
 * FFT kernels, 0 = automatic (for nphi = 3 * 2^k up to 3072: persistent CTAs
 * that prefetch their next latitude tile with tensor copies while the current
 * one is transformed, and on theta-contiguous grids write whole synthesis
 * tiles with tensor stores; phi-contiguous analysis keeps the direct
 * kernels), 1 = always the generic mixed-radix kernels, 2 = the fused
 * kernels without prefetch, 3 = prefetched loads with per-thread stores.
 * Option 6 (get only): FFT kernels of the last launch in this process, 0
 * generic, 1 fused direct, 2 prefetched.  Option 7 (test hook, default 0):
 * bytes, a multiple of 16 up to 4096, that the prefetching FFT kernels wait
 * for beyond what their tensor copies bring; a positive value makes their
 * bounded wait (about one second) give up, so that tests can check the error
 * path (shtns_b200_kernel_errors returns 1, no output is written).  Option 9
 * (test hook, set only, any plan): fills the static scratch array of
 * cu_SH_to_spat_noalloc on the current device with the byte value 0..255
 * (0xFF: NaN doubles) and waits for it.  Option 10: FP64 Legendre values
 * of the 64 x 64 tile synthesis, 0 (default) from a table of Y_k(theta)
 * built on the device on first use when it takes at most a quarter of the
 * free device memory and 8 GiB (about 0.2 GB at lmax 511 on 768 latitudes;
 * otherwise, and inside a stream capture before the table exists, on the
 * fly), 1 always on the fly, 2 always the table (an error when it does not
 * fit).  Both forms give bit-identical results; clones use the table of
 * their base plan.  Return 0 or -1.
 * No counterpart in SHTns 3.5.2. */
int shtns_b200_set_option(shtns_cfg, int option, int value);
int shtns_b200_get_option(shtns_cfg, int option);

/* Option 5 of shtns_b200_set_option: shape of the FP64 Legendre tiles, warps
 * along the rows: 1 = 32 rows x 128 columns, 2 = 64 x 64, 4 = 128 x 32,
 * 8 = SIMT kernels (FP64 FMA, recurrence in registers; calls with 1 to 4
 * field-components, others fall back to the automatic choice); 0 (default)
 * picks the SIMT kernels for at most 4 field-components in the synthesis and
 * 3 in the analysis, 128 x 32 for calls with at most 32 GEMM columns (8
 * field-components) and 64 x 64 otherwise.  Plan groups always use 64 x 64.
 * Option 4 of shtns_b200_set_option: split-precision Legendre stages with 3
 * to 7 balanced 8-bit digits per operand (products summed exactly; the
 * result carries about 8 x digits - 2 bits relative to the row and column
 * maxima; 7 digits stay within 1e-11 of FP64 at lmax 4095); 0 (default)
 * keeps the FP64 contraction.  Option 8 picks the form: 0 (default) a table
 * of the Legendre values as INT8 digits, built on the device on first use
 * (digits x 128-row x 128-step blocks over the orders, latitude tiles at or
 * beyond the polar threshold: about 69 GB for 7 digits at lmax 4095 on
 * 6144 latitudes) and contracted on the INT8 tensor cores with INT32
 * accumulation, synthesis and analysis, whole transforms with mres = 1;
 * 1: synthesis only, slices regenerated on the fly and contracted on the
 * FP16 tensor cores (analysis in FP64).  Clones use the table of their
 * base plan.
 * shtns_b200_kernel_errors waits for the device; returns 1 (and clears it)
 * if a bounded wait of a split-precision kernel or of the prefetching FFT
 * kernels gave up since the last call, else 0.
 * shtns_b200_split_table_bytes: bytes of the plan's digit table (0 when
 * none has been built).
 * No counterpart in SHTns 3.5.2. */
int shtns_b200_kernel_errors(shtns_cfg);
size_t shtns_b200_split_table_bytes(shtns_cfg);

/* Plan groups: transforms of fields of different lmax (scalar, and the vector
 * forms below), each on the grid
 * of its own plan, with the Legendre stage of all plans in one persistent
 * launch whose CTAs take work items (plan, order, tile) from a queue in
 * decreasing cost order.  Qlm[i] / Vr[i] hold nfields[i] contiguous fields of
 * plan i (device pointers; spec_dist = nlm, spat_dist = nspat of that plan).
 * All launches go to the compute stream of the first plan, so a call can be
 * captured in a CUDA graph (after one call with the same field counts, which
 * allocates the work buffers and the work list).  Plans in a group get a
 * common checkpoint spacing.  No counterpart in SHTns 3.5.2. */
typedef struct shtns_b200_group* shtns_group;
shtns_group shtns_b200_group_create(int nplans, shtns_cfg* plans);
void shtns_b200_group_destroy(shtns_group);
/* option 1: work order, 0 by decreasing cost (default), 1 plan/order/tile;
 * option 2: CTAs of the persistent launch per SM, 1-3 (0: 3);
 * option 3: checkpoint spacing of all plans, 8, 16 or 32;
 * option 4: 1 (default) the per-plan prologue, FFT and epilogue launches run
 * concurrently on side streams of the group (forked from and joined back
 * into the first plan's stream by events), 0 all on the first plan's stream;
 * option 5: Legendre stage, 0 (default) one persistent launch over all plans,
 * 1 each plan's own launch (its tile shape or SIMT kernels), chained with
 * the plan's prologue and FFT on its side stream (with option 4 = 1 the
 * plans run concurrently).  Return 0 or -1. */
int shtns_b200_group_set_option(shtns_group, int option, int value);
void shtns_b200_group_synth(shtns_group, cplx **Qlm, double **Vr, const int *nfields, int ltr);
void shtns_b200_group_analys(shtns_group, double **Vr, cplx **Qlm, const int *nfields, int ltr);
/* Vector transforms of a group (the plans' SHsphtor / SHqst forms): per plan
 * i, nfields[i] fields of each component, device pointers, as above. */
void shtns_b200_group_SHsphtor_to_spat(shtns_group, cplx **Slm, cplx **Tlm, double **Vt, double **Vp,
                                       const int *nfields, int ltr);
void shtns_b200_group_spat_to_SHsphtor(shtns_group, double **Vt, double **Vp, cplx **Slm, cplx **Tlm,
                                       const int *nfields, int ltr);
void shtns_b200_group_SHqst_to_spat(shtns_group, cplx **Qlm, cplx **Slm, cplx **Tlm, double **Vr, double **Vt,
                                    double **Vp, const int *nfields, int ltr);
void shtns_b200_group_spat_to_SHqst(shtns_group, double **Vr, double **Vt, double **Vp, cplx **Qlm, cplx **Slm,
                                    cplx **Tlm, const int *nfields, int ltr);

/* Scalar synthesis (same result as cu_SH_to_spat on device pointers) that
 * allocates no device memory, for callers that cannot call cudaMalloc where
 * they transform.  Its scratch is one static device array of 32 MiB that
 * every GPU loading this library holds until the process exits; plan and
 * batch must need at most that much (coefficient buffer + Fourier buffer,
 * e.g. one field up to lmax=511 on 768x1536), larger requests are rejected
 * with an error (shtns_b200_status() == 1) and nothing is written, as are
 * plans with split-precision synthesis (option 4) on.  Plan options 1, 3 and
 * 5 apply as in cu_SH_to_spat.  The
 * first call on a device resolves the array's address (and may load this
 * library's device code): make it before any stream capture.  All calls
 * share the array, so calls that overlap on the GPU race and must be
 * serialised by the caller.  Asynchronous on the plan's compute stream.
 * No counterpart in the reference. */
void cu_SH_to_spat_noalloc(shtns_cfg, cplx *Qlm, double *Vr, int ltr);

/* Order-split stages: one transform divided over processes (GPUs) by order.
 * Synthesis: each process runs shtns_b200_legendre_synth for its orders
 * m0..m1 over every grid row, the processes exchange Fourier rows (an
 * all-to-all) so that each holds every order of its block of grid rows, and
 * each runs shtns_b200_fourier_synth on its block.  Analysis runs
 * shtns_b200_fourier_analys on the block, the exchange backwards, and
 * shtns_b200_legendre_analys for the orders.  kind: 0 scalar (Q), 1
 * spheroidal/toroidal (S, T; outputs theta, phi components), 2 Q, S, T.
 * Fourier buffers (complex): on the Legendre side F[fc][im - m0][row] for the
 * nlat grid rows; on the Fourier side F[fc][im][r] for im = 0..mmax and the
 * nrows rows of the block (nrows even), fc = c * howmany + f for component c
 * of field f (shtns_set_batch).  Spatial blocks hold nrows consecutive grid
 * rows of each field in the plan's layout with nrows in place of nlat, fields
 * nphi*nrows doubles apart.  Spectral arrays keep the full layout (field
 * stride spec_dist); only orders m0..m1 are read or written.  Orders above
 * ltr are not written on the Fourier side (nor read by the FFT); the Legendre
 * analysis writes them as zero.  Device pointers; asynchronous on the plan's
 * compute stream.  No counterpart in SHTns 3.5.2 (single-process only). */
void shtns_b200_legendre_synth(shtns_cfg, int kind, cplx *Qlm, cplx *Slm, cplx *Tlm, cplx *F, int m0, int m1, int ltr);
void shtns_b200_fourier_synth(shtns_cfg, int kind, cplx *F, double *V0, double *V1, double *V2, int nrows, int ltr);
void shtns_b200_fourier_analys(shtns_cfg, int kind, double *V0, double *V1, double *V2, cplx *F, int nrows, int ltr);
void shtns_b200_legendre_analys(shtns_cfg, int kind, cplx *F, cplx *Qlm, cplx *Slm, cplx *Tlm, int m0, int m1, int ltr);

/* The order-split Legendre stages with the exchange fused in: the synthesis
 * stores Fourier row `row` of order im and field-component fc into the buffer
 * F[b] of the block b with lat0[b] <= row < lat0[b+1], at
 * (fc * (mmax+1) + im) * (lat0[b+1] - lat0[b]) + row - lat0[b] (the Fourier
 * side of shtns_b200_fourier_synth for that block); the analysis loads the
 * rows from there.  lat0[0] = 0, lat0[nblk] = nlat, 1 <= nblk <= 16.  The
 * buffers may be other GPUs' memory mapped with shtns_b200_ipc_open: the
 * rows then cross NVLink inside the Legendre kernels.  The caller orders
 * the stages across processes (a barrier between a rank's Legendre stage and
 * the FFT stages that read or write the same buffers).  No counterpart in
 * SHTns 3.5.2. */
void shtns_b200_legendre_synth_rows(shtns_cfg, int kind, cplx *Qlm, cplx *Slm, cplx *Tlm, int m0, int m1, int ltr,
                                    int nblk, const int *lat0, cplx **F);
void shtns_b200_legendre_analys_rows(shtns_cfg, int kind, int nblk, const int *lat0, cplx **F,
                                     cplx *Qlm, cplx *Slm, cplx *Tlm, int m0, int m1, int ltr);
/* Buffers for those stages: device allocations of their own (so that an IPC
 * handle maps exactly the buffer), the 64-byte CUDA IPC handle of such an
 * allocation (returns 0 or -1), the mapping of another process's handle
 * (NULL on error) and its release. */
void *shtns_b200_alloc(size_t bytes);
void shtns_b200_free(void *ptr);
int shtns_b200_ipc_handle(void *dev_ptr, void *handle64);
void *shtns_b200_ipc_open(const void *handle64);
void shtns_b200_ipc_close(void *ptr);

/* Batched point evaluation on device arrays: v[i] = the scalar field Qlm at
 * (cost[i], phi[i]) for i < npts (SHqst form: the three components of
 * SHqst_to_point).  One CTA per point; asynchronous on the plan's compute
 * stream; no grid needed.  Single points: SH_to_point / SHqst_to_point
 * (shtns.h).  No counterpart in SHTns 3.5.2. */
void shtns_b200_SH_to_points(shtns_cfg, cplx *Qlm, const double *cost, const double *phi, double *v, int npts);
void shtns_b200_SHqst_to_points(shtns_cfg, cplx *Qlm, cplx *Slm, cplx *Tlm, const double *cost, const double *phi,
                                double *vr, double *vt, double *vp, int npts);

#ifdef __cplusplus
}
#endif

#endif /* SHTNS_B200_EXT_H */
