/*
 * fftw_shim.c -- project-written implementation of the subset of the FFTW 3.3
 * API that the SHTns 3.5.2 CPU sources call.  TEST INFRASTRUCTURE ONLY: it is
 * linked into the reference CPU library built under oracle/_ref (the parity
 * checker and the timed CPU baseline).  Nothing in the shtns_b200 product
 * links or loads it.
 *
 * libfftw3 is not installed on the build or GPU machines.  SHTns uses FFTW
 * through these entry points (the call sites are in the reference's
 * sht_init.c:353-518 planFFT, sht_legendre.c:868-935, sht_func.c:84-88,762-876,
 * sht_odd_nlat.c and the SHT/*.gen.c drivers):
 *   fftw_plan_many_dft, fftw_plan_many_dft_r2c, fftw_plan_many_dft_c2r,
 *   fftw_plan_guru_split_dft, fftw_plan_dft_c2r_1d, fftw_execute_dft,
 *   fftw_execute_split_dft, fftw_execute_dft_r2c, fftw_execute_dft_c2r,
 *   fftw_destroy_plan, fftw_malloc, fftw_free, the wisdom file functions and
 *   the thread functions.
 *
 * Conventions follow FFTW's documentation: transforms are unnormalised, the
 * complex transform computes y[k] = sum_j x[j] exp(sign*2*pi*i*j*k/n) with
 * sign = FFTW_FORWARD (-1) or FFTW_BACKWARD (+1); r2c uses sign -1 and keeps
 * n/2+1 outputs; c2r uses sign +1 on Hermitian input; the split-array guru
 * transform is always the forward (-1) transform.
 *
 * Algorithm: recursive mixed-radix decimation in time (radix 4, 2, 3, 5 and a
 * direct DFT for any remaining prime factor), run on a block of up to VB
 * transforms at once with the block index innermost so the butterflies
 * vectorise.  The howmany loop is split over OpenMP threads when the plan was
 * made after fftw_plan_with_nthreads(n>1), as libfftw3_omp does.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <complex.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "fftw3/fftw3.h"

#define VB 8   /* transforms processed together (innermost, contiguous) */
#define MAXF 64

typedef struct { double re, im; } cpx;

typedef enum { K_DFT, K_SPLIT, K_R2C, K_C2R } kind_t;

struct fftw_plan_s {
	kind_t kind;
	int n;              /* transform length */
	int sign;           /* -1 or +1 */
	int howmany;
	long is, os;        /* element strides within one transform */
	long idist, odist;  /* distance between transforms */
	int nthreads;
	int nf;             /* number of factors */
	int fac[MAXF];
	cpx *tw;            /* twiddles, all levels concatenated */
	long twoff[MAXF];   /* offset of each level's twiddles */
	/* default arrays given at planning time (for fftw_execute) */
	void *in0, *in1, *out0, *out1;
};

static int g_nthreads = 1;

/* ---------- planning helpers ---------- */

static int factorize(int n, int *f)
{
	int nf = 0;
	while (n % 4 == 0) { f[nf++] = 4; n /= 4; }
	while (n % 2 == 0) { f[nf++] = 2; n /= 2; }
	while (n % 3 == 0) { f[nf++] = 3; n /= 3; }
	while (n % 5 == 0) { f[nf++] = 5; n /= 5; }
	for (int p = 7; (long)p * p <= n; p += 2)
		while (n % p == 0) { f[nf++] = p; n /= p; }
	if (n > 1) f[nf++] = n;
	return nf;
}

/* exp(sign*2*pi*i*k/n) with the angle reduced to [0, pi/4] for accuracy */
static cpx unit_root(long k, long n, int sign)
{
	k %= n; if (k < 0) k += n;
	/* use long double for the angle, symmetric reductions keep error ~1 ulp */
	long double a = 2.0L * 3.141592653589793238462643383279502884L * (long double)k / (long double)n;
	cpx w;
	w.re = (double) cosl(a);
	w.im = (double) (sign * sinl(a));
	return w;
}

static void plan_factors(struct fftw_plan_s *p)
{
	p->nf = factorize(p->n, p->fac);
	/* level j handles length L_j = n / (f_0*...*f_{j-1}), radix r = f_j, m = L_j/r */
	long tot = 0, L = p->n;
	for (int j = 0; j < p->nf; j++) {
		int r = p->fac[j];
		long m = L / r;
		p->twoff[j] = tot;
		tot += (long)(r - 1) * m + r;     /* twiddles + radix roots */
		L = m;
	}
	p->tw = (cpx *) malloc(sizeof(cpx) * (tot + 1));
	L = p->n;
	for (int j = 0; j < p->nf; j++) {
		int r = p->fac[j];
		long m = L / r;
		cpx *t = p->tw + p->twoff[j];
		for (int q = 1; q < r; q++)
			for (long k = 0; k < m; k++)
				t[(q - 1) * m + k] = unit_root((long)q * k, L, p->sign);
		cpx *rr = t + (long)(r - 1) * m;
		for (int q = 0; q < r; q++) rr[q] = unit_root(q, r, p->sign);
		L = m;
	}
}

/* ---------- execution on a block of nb (<=VB) transforms ----------
 * Data element j of transform b lives at buf[j*VB + b]. */

static void fft_rec(const struct fftw_plan_s *p, int lev, long n, const cpx *in, long istr,
                    cpx *out, int nb)
{
	if (n == 1) {
		for (int b = 0; b < nb; b++) out[b] = in[b];
		return;
	}
	const int r = p->fac[lev];
	const long m = n / r;
	for (int q = 0; q < r; q++)
		fft_rec(p, lev + 1, m, in + (long)q * istr * VB, istr * r, out + (long)q * m * VB, nb);
	const cpx *tw = p->tw + p->twoff[lev];
	const cpx *rr = tw + (long)(r - 1) * m;
	const double s = (double) p->sign;
	if (r == 2) {
		for (long k = 0; k < m; k++) {
			cpx w = tw[k];
			cpx *a = out + k * VB, *c = out + (k + m) * VB;
			for (int b = 0; b < nb; b++) {
				double tr = c[b].re * w.re - c[b].im * w.im;
				double ti = c[b].re * w.im + c[b].im * w.re;
				c[b].re = a[b].re - tr;  c[b].im = a[b].im - ti;
				a[b].re += tr;           a[b].im += ti;
			}
		}
	} else if (r == 4) {
		for (long k = 0; k < m; k++) {
			cpx w1 = tw[k], w2 = tw[m + k], w3 = tw[2 * m + k];
			cpx *x0 = out + k * VB, *x1 = out + (k + m) * VB, *x2 = out + (k + 2 * m) * VB, *x3 = out + (k + 3 * m) * VB;
			for (int b = 0; b < nb; b++) {
				double a0r = x0[b].re, a0i = x0[b].im;
				double a1r = x1[b].re * w1.re - x1[b].im * w1.im, a1i = x1[b].re * w1.im + x1[b].im * w1.re;
				double a2r = x2[b].re * w2.re - x2[b].im * w2.im, a2i = x2[b].re * w2.im + x2[b].im * w2.re;
				double a3r = x3[b].re * w3.re - x3[b].im * w3.im, a3i = x3[b].re * w3.im + x3[b].im * w3.re;
				double t0r = a0r + a2r, t0i = a0i + a2i, t1r = a0r - a2r, t1i = a0i - a2i;
				double t2r = a1r + a3r, t2i = a1i + a3i, t3r = a1r - a3r, t3i = a1i - a3i;
				/* multiply t3 by sign*i */
				double u3r = -s * t3i, u3i = s * t3r;
				x0[b].re = t0r + t2r;  x0[b].im = t0i + t2i;
				x2[b].re = t0r - t2r;  x2[b].im = t0i - t2i;
				x1[b].re = t1r + u3r;  x1[b].im = t1i + u3i;
				x3[b].re = t1r - u3r;  x3[b].im = t1i - u3i;
			}
		}
	} else if (r == 3) {
		const double c1 = -0.5, s1 = s * 0.86602540378443864676372317075294;
		for (long k = 0; k < m; k++) {
			cpx w1 = tw[k], w2 = tw[m + k];
			cpx *x0 = out + k * VB, *x1 = out + (k + m) * VB, *x2 = out + (k + 2 * m) * VB;
			for (int b = 0; b < nb; b++) {
				double a0r = x0[b].re, a0i = x0[b].im;
				double a1r = x1[b].re * w1.re - x1[b].im * w1.im, a1i = x1[b].re * w1.im + x1[b].im * w1.re;
				double a2r = x2[b].re * w2.re - x2[b].im * w2.im, a2i = x2[b].re * w2.im + x2[b].im * w2.re;
				double tr = a1r + a2r, ti = a1i + a2i;
				double dr = a1r - a2r, di = a1i - a2i;
				double mr = a0r + c1 * tr, mi = a0i + c1 * ti;
				x0[b].re = a0r + tr;  x0[b].im = a0i + ti;
				x1[b].re = mr - s1 * di;  x1[b].im = mi + s1 * dr;
				x2[b].re = mr + s1 * di;  x2[b].im = mi - s1 * dr;
			}
		}
	} else {
		/* generic radix: direct DFT of size r on twiddled inputs */
		cpx tmp[64 * VB];
		cpx *t = (r <= 64) ? tmp : (cpx *) malloc(sizeof(cpx) * r * VB);
		for (long k = 0; k < m; k++) {
			for (int q = 0; q < r; q++) {
				cpx w = (q == 0) ? (cpx){1.0, 0.0} : tw[(q - 1) * m + k];
				const cpx *x = out + (k + q * m) * VB;
				for (int b = 0; b < nb; b++) {
					t[q * VB + b].re = x[b].re * w.re - x[b].im * w.im;
					t[q * VB + b].im = x[b].re * w.im + x[b].im * w.re;
				}
			}
			for (int pp = 0; pp < r; pp++) {
				cpx *y = out + (k + pp * m) * VB;
				for (int b = 0; b < nb; b++) { y[b].re = 0.0; y[b].im = 0.0; }
				for (int q = 0; q < r; q++) {
					cpx w = rr[((long)q * pp) % r];
					for (int b = 0; b < nb; b++) {
						y[b].re += t[q * VB + b].re * w.re - t[q * VB + b].im * w.im;
						y[b].im += t[q * VB + b].re * w.im + t[q * VB + b].im * w.re;
					}
				}
			}
		}
		if (t != tmp) free(t);
	}
}

/* ---------- aliasing ----------
 * FFTW plans may be in place with different input and output layouts (the
 * reference's rotation FFT is an r2c of howmany transforms at stride howmany
 * with idist = odist = 1, in == out).  The block loops above write a block's
 * outputs before later blocks have read their inputs, so whenever the input
 * and output spans overlap (and the layouts are not identical), every input
 * is first gathered into a scratch array, as FFTW itself buffers such plans. */

/* [lo, hi) byte span of elements (j, t), j < n, t < howmany, at
 * base + (j*stride + t*dist)*elem bytes (strides may be negative). */
static void span(const void *base, long n, long stride, long howmany, long dist, long elem,
                 const char **lo, const char **hi)
{
	long a = 0, b = 0;
	long js = (n - 1) * stride, ts = (howmany - 1) * dist;
	if (js < 0) a += js; else b += js;
	if (ts < 0) a += ts; else b += ts;
	*lo = (const char *) base + a * elem;
	*hi = (const char *) base + (b + 1) * elem;
}

static int spans_overlap(const void *in, long ni, long is, long idist, long ielem,
                         const void *out, long no, long os, long odist, long oelem, long howmany)
{
	const char *il, *ih, *ol, *oh;
	span(in, ni, is, howmany, idist, ielem, &il, &ih);
	span(out, no, os, howmany, odist, oelem, &ol, &oh);
	return il < oh && ol < ih;
}

/* Run transforms [t0, t1) of a complex plan; input/output element (j, t) is at
 * base + j*stride + t*dist, given as separate real and imaginary pointers with a
 * step of 2 doubles for interleaved complex data or 1 for split arrays. */
static void run_block(const struct fftw_plan_s *p, long t0, long t1,
                      const double *ir, const double *ii, long istep_re_im_stride, long is, long idist,
                      double *orr, double *oi, long os, long odist, cpx *bin, cpx *bout)
{
	const long n = p->n;
	for (long t = t0; t < t1; t += VB) {
		int nb = (int)((t1 - t < VB) ? (t1 - t) : VB);
		for (long j = 0; j < n; j++)
			for (int b = 0; b < nb; b++) {
				long o = j * is + (t + b) * idist;
				bin[j * VB + b].re = ir[o * istep_re_im_stride];
				bin[j * VB + b].im = ii[o * istep_re_im_stride];
			}
		fft_rec(p, 0, n, bin, 1, bout, nb);
		for (long j = 0; j < n; j++)
			for (int b = 0; b < nb; b++) {
				long o = j * os + (t + b) * odist;
				orr[o * istep_re_im_stride] = bout[j * VB + b].re;
				oi[o * istep_re_im_stride] = bout[j * VB + b].im;
			}
	}
}

/* Generic complex execution.  step = 2 for interleaved complex arrays (real part
 * at 2*o, imag at 2*o+1), 1 for split arrays.  All reads of a block finish
 * before its writes, and blocks touch disjoint transforms, so in-place plans
 * with equal layouts run directly; other overlapping plans are gathered first. */
static void exec_complex(const struct fftw_plan_s *p, const double *ir, const double *ii,
                         double *orr, double *oi, long step)
{
	const long nblk = (p->howmany + VB - 1) / VB;
	const long n = p->n;
	const int same_layout = (ir == orr && ii == oi && p->is == p->os && p->idist == p->odist);
	if (!same_layout &&
	    (spans_overlap(ir, n, p->is * step, p->idist * step, 8, orr, n, p->os * step, p->odist * step, 8, p->howmany) ||
	     spans_overlap(ir, n, p->is * step, p->idist * step, 8, oi, n, p->os * step, p->odist * step, 8, p->howmany) ||
	     spans_overlap(ii, n, p->is * step, p->idist * step, 8, orr, n, p->os * step, p->odist * step, 8, p->howmany) ||
	     spans_overlap(ii, n, p->is * step, p->idist * step, 8, oi, n, p->os * step, p->odist * step, 8, p->howmany))) {
		/* gather all inputs (same re/im step as the output), then run from the copy */
		const long tot = n * (long) p->howmany;
		double *g = (double *) malloc(sizeof(double) * 2 * tot);
		double *gr = g, *gi = (step == 2) ? g + 1 : g + tot;
		for (long t = 0; t < p->howmany; t++)
			for (long j = 0; j < n; j++) {
				long o = j * p->is + t * p->idist, d = j + t * n;
				gr[d * step] = ir[o * step];
				gi[d * step] = ii[o * step];
			}
		struct fftw_plan_s q = *p;
		q.is = 1; q.idist = n;
		exec_complex(&q, gr, gi, orr, oi, step);
		free(g);
		return;
	}
	int nth = p->nthreads;
#ifdef _OPENMP
	if (omp_in_parallel()) nth = 1;
	if (nth > nblk) nth = (int) nblk;
	if (nth < 1) nth = 1;
	#pragma omp parallel num_threads(nth) if(nth > 1)
#endif
	{
		cpx *bin = (cpx *) malloc(sizeof(cpx) * n * VB);
		cpx *bout = (cpx *) malloc(sizeof(cpx) * n * VB);
#ifdef _OPENMP
		#pragma omp for schedule(static)
#endif
		for (long blk = 0; blk < nblk; blk++) {
			long t0 = blk * VB, t1 = t0 + VB;
			if (t1 > p->howmany) t1 = p->howmany;
			run_block(p, t0, t1, ir, ii, step, p->is, p->idist, orr, oi, p->os, p->odist, bin, bout);
		}
		free(bin); free(bout);
	}
}

/* ---------- public API ---------- */

static struct fftw_plan_s *new_plan(kind_t kind, int n, int sign, int howmany,
                                    long is, long idist, long os, long odist)
{
	struct fftw_plan_s *p = (struct fftw_plan_s *) calloc(1, sizeof(*p));
	p->kind = kind; p->n = n; p->sign = sign; p->howmany = howmany;
	p->is = is; p->os = os; p->idist = idist; p->odist = odist;
	p->nthreads = g_nthreads;
	plan_factors(p);
	return p;
}

static void need_rank1(int rank, const char *who)
{
	if (rank != 1) { fprintf(stderr, "fftw_shim: %s supports rank 1 only\n", who); abort(); }
}

fftw_plan fftw_plan_many_dft(int rank, const int *n, int howmany,
                             fftw_complex *in, const int *inembed, int istride, int idist,
                             fftw_complex *out, const int *onembed, int ostride, int odist,
                             int sign, unsigned flags)
{
	(void) inembed; (void) onembed; (void) flags;
	need_rank1(rank, "fftw_plan_many_dft");
	struct fftw_plan_s *p = new_plan(K_DFT, n[0], sign, howmany, istride, idist, ostride, odist);
	p->in0 = in; p->out0 = out;
	return p;
}

fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany,
                                 double *in, const int *inembed, int istride, int idist,
                                 fftw_complex *out, const int *onembed, int ostride, int odist,
                                 unsigned flags)
{
	(void) inembed; (void) onembed; (void) flags;
	need_rank1(rank, "fftw_plan_many_dft_r2c");
	struct fftw_plan_s *p = new_plan(K_R2C, n[0], FFTW_FORWARD, howmany, istride, idist, ostride, odist);
	p->in0 = in; p->out0 = out;
	return p;
}

fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany,
                                 fftw_complex *in, const int *inembed, int istride, int idist,
                                 double *out, const int *onembed, int ostride, int odist,
                                 unsigned flags)
{
	(void) inembed; (void) onembed; (void) flags;
	need_rank1(rank, "fftw_plan_many_dft_c2r");
	struct fftw_plan_s *p = new_plan(K_C2R, n[0], FFTW_BACKWARD, howmany, istride, idist, ostride, odist);
	p->in0 = in; p->out0 = out;
	return p;
}

fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *in, double *out, unsigned flags)
{
	int nn = n;
	return fftw_plan_many_dft_c2r(1, &nn, 1, in, NULL, 1, n / 2 + 1, out, NULL, 1, n, flags);
}

fftw_plan fftw_plan_guru_split_dft(int rank, const fftw_iodim *dims,
                                   int howmany_rank, const fftw_iodim *howmany_dims,
                                   double *ri, double *ii, double *ro, double *io,
                                   unsigned flags)
{
	(void) flags;
	need_rank1(rank, "fftw_plan_guru_split_dft");
	int howmany = 1; long idist = 0, odist = 0;
	if (howmany_rank == 1) { howmany = howmany_dims[0].n; idist = howmany_dims[0].is; odist = howmany_dims[0].os; }
	else if (howmany_rank != 0) { fprintf(stderr, "fftw_shim: howmany_rank > 1 unsupported\n"); abort(); }
	struct fftw_plan_s *p = new_plan(K_SPLIT, dims[0].n, FFTW_FORWARD, howmany, dims[0].is, idist, dims[0].os, odist);
	p->in0 = ri; p->in1 = ii; p->out0 = ro; p->out1 = io;
	return p;
}

void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out)
{
	double *i = (double *) in, *o = (double *) out;
	exec_complex(p, i, i + 1, o, o + 1, 2);
}

void fftw_execute_split_dft(const fftw_plan p, double *ri, double *ii, double *ro, double *io)
{
	exec_complex(p, ri, ii, ro, io, 1);
}

/* r2c: widen the real input to complex, transform, keep n/2+1 outputs. */
void fftw_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out)
{
	const long n = p->n, nc = n / 2 + 1;
	if (spans_overlap(in, n, p->is, p->idist, 8, out, nc, p->os, p->odist, 16, p->howmany)) {
		const long tot = n * (long) p->howmany;
		double *g = (double *) malloc(sizeof(double) * tot);
		for (long t = 0; t < p->howmany; t++)
			for (long j = 0; j < n; j++) g[j + t * n] = in[j * p->is + t * p->idist];
		struct fftw_plan_s q = *p;
		q.is = 1; q.idist = n;
		fftw_execute_dft_r2c(&q, g, out);
		free(g);
		return;
	}
	cpx *bin = (cpx *) malloc(sizeof(cpx) * n * VB);
	cpx *bout = (cpx *) malloc(sizeof(cpx) * n * VB);
	double *o = (double *) out;
	for (long t = 0; t < p->howmany; t += VB) {
		int nb = (int)((p->howmany - t < VB) ? (p->howmany - t) : VB);
		for (long j = 0; j < n; j++)
			for (int b = 0; b < nb; b++) {
				bin[j * VB + b].re = in[j * p->is + (t + b) * p->idist];
				bin[j * VB + b].im = 0.0;
			}
		fft_rec(p, 0, n, bin, 1, bout, nb);
		for (long k = 0; k < nc; k++)
			for (int b = 0; b < nb; b++) {
				long q = k * p->os + (t + b) * p->odist;
				o[2 * q] = bout[k * VB + b].re;
				o[2 * q + 1] = bout[k * VB + b].im;
			}
	}
	free(bin); free(bout);
}

/* c2r: rebuild the full Hermitian spectrum, transform with sign +1, keep the
 * real part.  FFTW ignores the imaginary parts of the k=0 and k=n/2 inputs. */
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out)
{
	const long n = p->n, nc = n / 2 + 1;
	if (spans_overlap(in, nc, p->is, p->idist, 16, out, n, p->os, p->odist, 8, p->howmany)) {
		const long tot = nc * (long) p->howmany;
		fftw_complex *g = (fftw_complex *) malloc(sizeof(fftw_complex) * tot);
		const double *x = (const double *) in;
		for (long t = 0; t < p->howmany; t++)
			for (long k = 0; k < nc; k++) {
				long q = k * p->is + t * p->idist;
				((double *) g)[2 * (k + t * nc)] = x[2 * q];
				((double *) g)[2 * (k + t * nc) + 1] = x[2 * q + 1];
			}
		struct fftw_plan_s q = *p;
		q.is = 1; q.idist = nc;
		fftw_execute_dft_c2r(&q, g, out);
		free(g);
		return;
	}
	cpx *bin = (cpx *) malloc(sizeof(cpx) * n * VB);
	cpx *bout = (cpx *) malloc(sizeof(cpx) * n * VB);
	const double *x = (const double *) in;
	for (long t = 0; t < p->howmany; t += VB) {
		int nb = (int)((p->howmany - t < VB) ? (p->howmany - t) : VB);
		for (long k = 0; k < nc; k++)
			for (int b = 0; b < nb; b++) {
				long q = k * p->is + (t + b) * p->idist;
				double re = x[2 * q], im = x[2 * q + 1];
				if (k == 0 || 2 * k == n) im = 0.0;
				bin[k * VB + b].re = re;  bin[k * VB + b].im = im;
				if (k > 0 && 2 * k != n) { bin[(n - k) * VB + b].re = re;  bin[(n - k) * VB + b].im = -im; }
			}
		fft_rec(p, 0, n, bin, 1, bout, nb);
		for (long j = 0; j < n; j++)
			for (int b = 0; b < nb; b++)
				out[j * p->os + (t + b) * p->odist] = bout[j * VB + b].re;
	}
	free(bin); free(bout);
}

void fftw_execute(const fftw_plan p)
{
	switch (p->kind) {
		case K_DFT:   fftw_execute_dft(p, (fftw_complex *) p->in0, (fftw_complex *) p->out0); break;
		case K_SPLIT: fftw_execute_split_dft(p, (double *) p->in0, (double *) p->in1, (double *) p->out0, (double *) p->out1); break;
		case K_R2C:   fftw_execute_dft_r2c(p, (double *) p->in0, (fftw_complex *) p->out0); break;
		case K_C2R:   fftw_execute_dft_c2r(p, (fftw_complex *) p->in0, (double *) p->out0); break;
	}
}

void fftw_destroy_plan(fftw_plan p)
{
	if (p) { free(p->tw); free(p); }
}

void *fftw_malloc(size_t n)
{
	void *ptr = NULL;
	if (posix_memalign(&ptr, 64, n ? n : 64) != 0) return NULL;
	return ptr;
}

void fftw_free(void *p) { free(p); }

/* Wisdom: the shim's plans carry no measured state, so there is nothing to
 * save or restore.  FFTW returns 0 when no wisdom was read. */
int fftw_import_wisdom_from_file(FILE *input_file) { (void) input_file; return 0; }
void fftw_export_wisdom_to_file(FILE *output_file) { (void) output_file; }

int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int nthreads) { g_nthreads = (nthreads > 0) ? nthreads : 1; }
void fftw_cleanup(void) {}
void fftw_cleanup_threads(void) {}
double fftw_cost(const fftw_plan p) { (void) p; return 0.0; }
void fftw_print_plan(const fftw_plan p)
{
	printf("(shim-dft n=%d howmany=%d radices:", p->n, p->howmany);
	for (int j = 0; j < p->nf; j++) printf(" %d", p->fac[j]);
	printf(")\n");
}
