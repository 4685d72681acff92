/*
 * A C99 caller of the drop-in boundary, in the manner of the reference's
 * cudamaxrelerror.cu (host transforms beside cu_* device transforms on the
 * same random grid data, round trips compared).  Built and run by
 * tests/test_c_callers_gpu.py against include/shtns.h, include/shtns_cuda.h
 * and libshtns_b200.so:
 *
 *   gcc -std=c99 -D_DEFAULT_SOURCE -I include -I <cuda>/include cu_roundtrip.c \
 *       -L shtns_b200 -lshtns_b200 -L <cuda>/lib64 -lcudart -lm
 *
 * Checks (normwise: max |a - b| / max |a|):
 *   1. host API: analysis then synthesis projects the grid onto degrees <= lmax;
 *      a second projection changes it by rounding only (<= 1e-12);
 *   2. cu_* API on device arrays gives the host API's spectra and grids (<= 1e-12)
 *      and the same idempotent round trip;
 *   3. cu_*_float on FP32 arrays agrees with the FP64 result to FP32 rounding;
 *   4. the public plan fields (nlm, lmax, nlat, nphi, ct) read from C.
 * Exit status 0 when every check passes.
 */
#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "shtns.h"
#include "shtns_cuda.h"

static double relerr(const double *a, const double *b, long n)
{
	double num = 0.0, den = 0.0;
	for (long i = 0; i < n; i++) {
		const double d = fabs(a[i] - b[i]);
		if (d > num) num = d;
		if (fabs(a[i]) > den) den = fabs(a[i]);
	}
	return den > 0.0 ? num / den : num;
}

static double relerr_f(const double *a, const float *b, long n)
{
	double num = 0.0, den = 0.0;
	for (long i = 0; i < n; i++) {
		const double d = fabs(a[i] - (double) b[i]);
		if (d > num) num = d;
		if (fabs(a[i]) > den) den = fabs(a[i]);
	}
	return den > 0.0 ? num / den : num;
}

static int failures = 0;

static void check(const char *what, double err, double tol)
{
	const int ok = err <= tol;
	printf("%-44s %.3e  %s\n", what, err, ok ? "OK" : "FAIL");
	if (!ok) failures++;
}

#define CUDA_OK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { \
	printf("CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); return 2; } } while (0)

int main(void)
{
	const int nlon = 480, nlat = 256, lmax = 150;
	const long nspat = (long) nlon * nlat;

	double *init_x = malloc(sizeof(double) * nspat);
	srand(1234);
	for (long i = 0; i < nspat; i++) init_x[i] = (1.0 * rand()) / RAND_MAX - 0.5;

	/* host API */
	shtns_cfg sht = shtns_create(lmax, lmax, 1, sht_orthonormal);
	if (shtns_set_grid(sht, sht_quick_init, 0.0, nlat, nlon) != (int) nspat) { printf("set_grid failed\n"); return 2; }
	if (sht->nlm != (unsigned) nlm_calc(lmax, lmax, 1) || sht->lmax != lmax || sht->nlat != (unsigned) nlat ||
	    sht->nphi != (unsigned) nlon || !(sht->ct[0] > sht->ct[nlat - 1])) {
		printf("public plan fields unexpected\n");
		return 2;
	}
	const long nlm = sht->nlm;
	double *x1 = malloc(sizeof(double) * nspat), *x2 = malloc(sizeof(double) * nspat);
	cplx *q = malloc(sizeof(cplx) * nlm), *q2 = malloc(sizeof(cplx) * nlm);
	memcpy(x1, init_x, sizeof(double) * nspat);
	spat_to_SH(sht, x1, q);        /* q: spectrum of the random grid */
	SH_to_spat(sht, q, x2);        /* x2: its projection onto degrees <= lmax */
	spat_to_SH(sht, x2, q2);
	SH_to_spat(sht, q2, x1);       /* x1: projection of the projection */
	check("host: projection is idempotent", relerr(x2, x1, nspat), 1e-12);
	check("host: spectrum of the projection", relerr((double *) q, (double *) q2, 2 * nlm), 1e-12);

	/* device API on a plan of its own */
	shtns_cfg gsht = shtns_create(lmax, lmax, 1, sht_orthonormal);
	shtns_set_grid(gsht, (enum shtns_type)(sht_quick_init | SHT_ALLOW_GPU), 0.0, nlat, nlon);
	double *d_x1, *d_x2;
	cplx *d_q;
	CUDA_OK(cudaMalloc((void **) &d_x1, sizeof(double) * nspat));
	CUDA_OK(cudaMalloc((void **) &d_x2, sizeof(double) * nspat));
	CUDA_OK(cudaMalloc((void **) &d_q, sizeof(cplx) * nlm));
	CUDA_OK(cudaMemcpy(d_x1, init_x, sizeof(double) * nspat, cudaMemcpyHostToDevice));
	double *hx1 = malloc(sizeof(double) * nspat), *hx2 = malloc(sizeof(double) * nspat);
	cplx *hq = malloc(sizeof(cplx) * nlm);
	cu_spat_to_SH(gsht, d_x1, d_q, lmax);
	CUDA_OK(cudaMemcpy(hq, d_q, sizeof(cplx) * nlm, cudaMemcpyDeviceToHost));
	cu_SH_to_spat(gsht, d_q, d_x2, lmax);
	CUDA_OK(cudaMemcpy(hx2, d_x2, sizeof(double) * nspat, cudaMemcpyDeviceToHost));
	cu_spat_to_SH(gsht, d_x2, d_q, lmax);
	cu_SH_to_spat(gsht, d_q, d_x1, lmax);
	CUDA_OK(cudaMemcpy(hx1, d_x1, sizeof(double) * nspat, cudaMemcpyDeviceToHost));
	check("cu_*: spectrum equals host spat_to_SH", relerr((double *) q, (double *) hq, 2 * nlm), 1e-12);
	check("cu_*: projection equals host SH_to_spat", relerr(x2, hx2, nspat), 1e-12);
	check("cu_*: projection is idempotent", relerr(hx2, hx1, nspat), 1e-12);

	/* FP32 device arrays (cu_*_float) */
	float *fx = malloc(sizeof(float) * nspat), *d_fx;
	cplx_f *d_fq;
	for (long i = 0; i < nspat; i++) fx[i] = (float) x2[i];
	CUDA_OK(cudaMalloc((void **) &d_fx, sizeof(float) * nspat));
	CUDA_OK(cudaMalloc((void **) &d_fq, sizeof(cplx_f) * nlm));
	CUDA_OK(cudaMemcpy(d_fx, fx, sizeof(float) * nspat, cudaMemcpyHostToDevice));
	cu_spat_to_SH_float(gsht, d_fx, d_fq, lmax);
	cu_SH_to_spat_float(gsht, d_fq, d_fx, lmax);
	CUDA_OK(cudaMemcpy(fx, d_fx, sizeof(float) * nspat, cudaMemcpyDeviceToHost));
	check("cu_*_float: FP32 round trip", relerr_f(x2, fx, nspat), 1e-6);

	cudaFree(d_x1); cudaFree(d_x2); cudaFree(d_q); cudaFree(d_fx); cudaFree(d_fq);
	shtns_destroy(gsht);
	shtns_destroy(sht);
	free(init_x); free(x1); free(x2); free(q); free(q2); free(hx1); free(hx2); free(hq); free(fx);
	printf(failures ? "FAILED: %d\n" : "ALL OK\n", failures);
	return failures ? 1 : 0;
}
