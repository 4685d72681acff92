// Local and partial evaluation of spherical-harmonic expansions on sm_100a:
// values at points (SH_to_point, SH_to_point_cplx, SH_to_grad_point,
// SHqst_to_point; sht_func.c:516-730), on one latitude (SH_to_lat,
// SHqst_to_lat; sht_func.c:732-885), associated Legendre arrays
// (legendre_sphPlm_array / _deriv_array, sht_legendre.c:238-440) and the
// l+-1 operators (SH_mul_mx, sht_func.c:484-507).  None needs a grid.
//
// Per order m, one thread runs the classic recurrence of the plan
// (P_l = a_l x P_{l-1} + b_l P_{l-2}, the alm table of shtns_create) on the
// pair y = P_l^m / sin(theta) (m > 0; P_l^0 for m = 0) and dy = dP_l^m/dtheta,
//   dy_l = a_l (x dy_{l-1} - s y_{l-1}) + b_l dy_{l-2},  s = sin^2 (m > 0), sin (m = 0),
// seeded with y_m = al[0] sin^(m-1) theta, dy_m = m x y_m, and sums the
// spectral coefficients of that order against y and dy.  The seed is formed
// as a mantissa times 2^E (binary powering with frexp) and the recurrence
// runs on the scaled values until they are significant (E folded back to 0),
// as in the checkpoint kernel; terms below 2^-100 are dropped, as the
// reference drops its scaled values (sht_legendre.c:383-404).
// The per-order results are the Fourier coefficients of the fields along
// the latitude:
//   F_r = sum_l y Q          (times sin(theta) for m > 0)
//   F_t = i m sum y T + sum dy S,   F_p = i m sum y S - sum dy T
// (m = 0: real parts only), and a field value is
//   v(phi) = sum_m (2 - delta_m0) Re(F_m e^{i m phi}).
#include "sht_internal.h"

#include <cstring>
#include <cstdint>
#include <cmath>
#include <vector>

namespace {

#define LOC_FOLD 600          // fold the exponent when E >= -LOC_FOLD
#define LOC_BIG 0x1p500       // rescale scaled values above this magnitude

struct LocalParams {
	const double* alm;        // classic recurrence per order: seed, a_{m+1}, then (b_l, a_l)
	const long* almoff;       // offset of each order in alm
	int lmax, mmax, mres, ltr, mtr;
	int cplx;                 // 1: Q holds a complex field in the LM_cplx layout (mres = 1)
	const double2 *Q, *S, *T; // spectral arrays (device, plan layout; any may be null)
	double2* F;               // per order: F[im], F[nm + im], F[2 nm + im] (r, theta, phi); cplx: F[im], F[nm + im] (+m, -m)
	int nm;                   // stride of F (mtr + 1)
	double* yl;               // Legendre arrays (lmax - m + 1 values each), or null
	double* dyl;
	int* lnz;                 // first degree with a stored non-zero value
};

__device__ __forceinline__ long lm_index(const LocalParams& p, int im, int l)     // LM(l, m), shtns.h:104-106
{
	return (long) im * (2 * p.lmax + 2 - (im + 1) * p.mres) / 2 + l;
}

__device__ __forceinline__ long lm_cplx_index(const LocalParams& p, int l, int m)  // LM_cplx(l, m), mres = 1
{
	return (l <= p.mmax) ? (long) l * (l + 1) + m : (long) p.mmax * (2 * l - p.mmax) + l + m;
}

__device__ __forceinline__ double2 cfma(double a, double2 z, double2 acc) { return make_double2(fma(a, z.x, acc.x), fma(a, z.y, acc.y)); }

// sums of order im at (x, st): Q against y, S and T against y and dy; for a
// complex field, Q(l, +m) and Q(l, -m) against y.  With yl set, the values
// are stored instead (Legendre arrays: P (deriv == 0) or P / sin and dP/dtheta).
struct OrderSums { double2 q, q2, sdt, tdt, sy, ty; };

__device__ OrderSums order_sums(const LocalParams& p, int im, double x, double st, int deriv)
{
	OrderSums r;
	r.q = r.q2 = r.sdt = r.tdt = r.sy = r.ty = make_double2(0.0, 0.0);
	const int m = im * p.mres;
	const double* al = p.alm + p.almoff[im];
	double s2 = st;
	double y0 = al[0], dy0 = 0.0;
	int E = 0;
	if (m > 0) {
		// sin^(m-1) = mantissa * 2^E
		double y = 1.0;
		int be, te;
		double b = frexp(st, &be);
		if (st == 0.0) { y = (m == 1) ? 1.0 : 0.0; }
		else {
			for (int n = m - 1; n; n >>= 1) {
				if (n & 1) { y = frexp(y * b, &te); E += be + te; }
				b = frexp(b * b, &te); be = 2 * be + te;
			}
		}
		y0 *= y;
		if (E >= -LOC_FOLD) { y0 = ldexp(y0, E); E = 0; }
		dy0 = x * m * y0;
		s2 = st * st;
	}
	double y1 = al[1] * (x * y0);
	double dy1 = al[1] * (x * dy0 - s2 * y0);
	int first = -1;
	auto put = [&](int l, double y, double dy) {
		if (p.yl) {
			const double v = E ? 0.0 : y;
			p.yl[l - m] = (deriv || m == 0) ? v : v * st;
			if (p.dyl) p.dyl[l - m] = E ? 0.0 : dy;
			if (!E && first < 0) first = l;
			return;
		}
		if (E) return;
		if (p.cplx) {
			r.q = cfma(y, p.Q[lm_cplx_index(p, l, m)], r.q);
			if (m > 0) r.q2 = cfma(y, p.Q[lm_cplx_index(p, l, -m)], r.q2);
			return;
		}
		const long j = lm_index(p, im, l);
		if (p.Q) r.q = cfma(y, p.Q[j], r.q);
		if (p.S) { const double2 v = p.S[j]; r.sdt = cfma(dy, v, r.sdt); r.sy = cfma(y, v, r.sy); }
		if (p.T) { const double2 v = p.T[j]; r.tdt = cfma(dy, v, r.tdt); r.ty = cfma(y, v, r.ty); }
	};
	if (m <= p.ltr) put(m, y0, dy0);
	if (m + 1 <= p.ltr) put(m + 1, y1, dy1);
	for (int l = m + 2; l <= p.ltr; l++) {
		const double b = al[2 * (l - m - 1)], a = al[2 * (l - m - 1) + 1];
		const double y2 = a * (x * y1) + b * y0;
		const double dy2 = a * (x * dy1 - s2 * y1) + b * dy0;
		y0 = y1; y1 = y2; dy0 = dy1; dy1 = dy2;
		if (E && fabs(y1) > LOC_BIG) {
			if (E >= -LOC_FOLD) {
				y0 = ldexp(y0, E); y1 = ldexp(y1, E); dy0 = ldexp(dy0, E); dy1 = ldexp(dy1, E); E = 0;
			} else {
				y0 *= 0x1p-500; y1 *= 0x1p-500; dy0 *= 0x1p-500; dy1 *= 0x1p-500; E += 500;
			}
		}
		put(l, y1, dy1);
	}
	if (p.lnz) *p.lnz = (first < 0) ? p.ltr + 1 : first;
	return r;
}

__device__ __forceinline__ double2 times_im(double m, double2 z) { return make_double2(-m * z.y, m * z.x); }

// Fourier coefficients of order im at (x, st)
__device__ void order_fourier(const LocalParams& p, int im, double x, double st, double2& fr, double2& ft, double2& fp)
{
	const OrderSums r = order_sums(p, im, x, st, 1);
	const int m = im * p.mres;
	if (p.cplx) {
		fr = r.q;
		const double sg = (m & 1) ? -1.0 : 1.0;        // (-1)^m for the order -m
		ft = make_double2(sg * r.q2.x, sg * r.q2.y);
		if (m > 0) { fr = make_double2(fr.x * st, fr.y * st); ft = make_double2(ft.x * st, ft.y * st); }
		fp = make_double2(0.0, 0.0);
		return;
	}
	if (m == 0) {
		fr = make_double2(r.q.x, 0.0);
		ft = make_double2(r.sdt.x, 0.0);
		fp = make_double2(-r.tdt.x, 0.0);
		return;
	}
	fr = make_double2(r.q.x * st, r.q.y * st);
	const double2 a = times_im((double) m, r.ty), b = times_im((double) m, r.sy);
	ft = make_double2(a.x + r.sdt.x, a.y + r.sdt.y);
	fp = make_double2(b.x - r.tdt.x, b.y - r.tdt.y);
}

// one latitude: Fourier coefficients of every order im <= mtr
__global__ void lat_coef_kernel(LocalParams p, double x, double st)
{
	const int im = blockIdx.x * blockDim.x + threadIdx.x;
	if (im > p.mtr) return;
	double2 fr, ft, fp;
	order_fourier(p, im, x, st, fr, ft, fp);
	p.F[im] = fr;
	p.F[p.nm + im] = ft;
	p.F[2 * p.nm + im] = fp;
}

// v_j = sum_m (2 - delta_m0) Re(F_m e^{2 pi i m j / nphi}), with the angle
// reduced exactly ((m j) mod nphi); ncomp components
__global__ void lat_dft_kernel(const double2* __restrict__ F, int nm, int mres, int nphi, int ncomp,
                               double* v0, double* v1, double* v2)
{
	const int j = blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= nphi) return;
	double acc[3] = {0.0, 0.0, 0.0};
	for (int im = 0; im < nm; im++) {
		const long mj = ((long) im * mres * j) % nphi;
		double sn, cs;
		sincospi(2.0 * (double) mj / (double) nphi, &sn, &cs);
		const double w = im ? 2.0 : 1.0;
		for (int c = 0; c < ncomp; c++) {
			const double2 f = F[c * nm + im];
			acc[c] = fma(w, f.x * cs - f.y * sn, acc[c]);
		}
	}
	double* out[3] = {v0, v1, v2};
	for (int c = 0; c < ncomp; c++) out[c][j] = acc[c];
}

// point values: block reduction of the orders' contributions.  mode 0: real
// fields (ncomp components), mode 1: complex field (sum F_m e^{im phi} +
// F'_m e^{-im phi}).  One CTA per point; orders are dealt to the threads in a
// snake order to balance the triangular work.
#define PT_THREADS 128

__device__ __forceinline__ int snake_order(int i, int nt)
{
	const int r = i / nt, c = i - r * nt;
	return (r & 1) ? r * nt + (nt - 1 - c) : i;
}

__global__ void __launch_bounds__(PT_THREADS) point_kernel(LocalParams p, const double* __restrict__ cost,
                                                           const double* __restrict__ phi, int ncomp, int mode,
                                                           double* o0, double* o1, double* o2)
{
	__shared__ double red[PT_THREADS / 32][6];
	const int pt = blockIdx.x;
	const double x = cost[pt], ph = phi[pt];
	const double st = sqrt((1.0 - x) * (1.0 + x));
	double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
	const int npad = (p.mtr + PT_THREADS) / PT_THREADS * PT_THREADS;    // orders rounded up to whole rows
	for (int i = threadIdx.x; i < npad; i += PT_THREADS) {
		const int im = snake_order(i, PT_THREADS);
		if (im > p.mtr) continue;
		double2 fr, ft, fp;
		order_fourier(p, im, x, st, fr, ft, fp);
		const double m = (double) im * p.mres;
		double sn, cs;
		sincos(m * ph, &sn, &cs);
		if (mode == 1) {
			// z = F e^{i m phi} + F' e^{-i m phi}
			acc[0] += fr.x * cs - fr.y * sn + (im ? ft.x * cs + ft.y * sn : 0.0);
			acc[1] += fr.x * sn + fr.y * cs + (im ? ft.y * cs - ft.x * sn : 0.0);
		} else {
			const double w = im ? 2.0 : 1.0;
			acc[0] += w * (fr.x * cs - fr.y * sn);
			acc[1] += w * (ft.x * cs - ft.y * sn);
			acc[2] += w * (fp.x * cs - fp.y * sn);
		}
	}
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	#pragma unroll
	for (int c = 0; c < 3; c++) {
		double v = acc[c];
		for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
		if (lane == 0) red[warp][c] = v;
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		double s[3] = {0.0, 0.0, 0.0};
		for (int w = 0; w < PT_THREADS / 32; w++)
			for (int c = 0; c < 3; c++) s[c] += red[w][c];
		if (mode == 1) { o0[2 * pt] = s[0]; o0[2 * pt + 1] = s[1]; }
		else {
			o0[pt] = s[0];
			if (ncomp > 1) { o1[pt] = s[1]; o2[pt] = s[2]; }
		}
	}
}

// associated Legendre values of every order im <= mmax at x, for degrees
// m..lmax, into out[ofs(m) + l - m], ofs(m) = m (lmax + 2) - m (m + 1) / 2
__global__ void plm_table_kernel(LocalParams p, double x, double st, double* out)
{
	const int im = blockIdx.x * blockDim.x + threadIdx.x;
	if (im > p.mmax) return;
	const int m = im * p.mres;
	LocalParams q = p;
	q.yl = out + (long) m * (p.lmax + 2) - (long) m * (m + 1) / 2;
	q.dyl = nullptr;
	q.lnz = nullptr;
	order_sums(q, im, x, st, 0);
}

__global__ void legendre_array_kernel(LocalParams p, int im, double x, double st, int deriv)
{
	if (threadIdx.x == 0 && blockIdx.x == 0) order_sums(p, im, x, st, deriv);
}

// R[lm] = mx[2 lm] Q[lm - 1] + mx[2 lm + 1] Q[lm + 1]
__global__ void mul_mx_kernel(const double* __restrict__ mx, const double2* __restrict__ Q, double2* __restrict__ R, long nlm)
{
	const long lm = (long) blockIdx.x * blockDim.x + threadIdx.x;
	if (lm >= nlm) return;
	double2 r = make_double2(0.0, 0.0);
	if (lm > 0) r = cfma(mx[2 * lm], Q[lm - 1], r);
	if (lm + 1 < nlm) r = cfma(mx[2 * lm + 1], Q[lm + 1], r);
	R[lm] = r;
}

// ---------------------------------------------------------------------------
bool loc_tables(shtns_cfg s)
{
	if (s->d_alm) return true;
	const size_t na = s->alm.size(), no = s->alm_off.size();
	void* d = nullptr;
	if (!shtb_cuda_ok(cudaMalloc(&d, sizeof(double) * na + sizeof(long) * no), "local evaluation tables")) return false;
	s->d_alm = static_cast<double*>(d);
	s->d_almoff = reinterpret_cast<long*>(s->d_alm + na);
	cudaMemcpy(s->d_alm, s->alm.data(), sizeof(double) * na, cudaMemcpyHostToDevice);
	cudaMemcpy(s->d_almoff, s->alm_off.data(), sizeof(long) * no, cudaMemcpyHostToDevice);
	return true;
}

void* loc_buf(shtns_cfg s, size_t bytes)
{
	if (s->loc_cap >= bytes && s->d_loc) return s->d_loc;
	if (s->d_loc) cudaFree(s->d_loc);
	s->d_loc = nullptr; s->loc_cap = 0;
	if (!shtb_cuda_ok(cudaMalloc(&s->d_loc, bytes), "local evaluation buffers")) { s->d_loc = nullptr; return nullptr; }
	s->loc_cap = bytes;
	return s->d_loc;
}

LocalParams loc_params(shtns_cfg s)
{
	LocalParams p;
	memset(&p, 0, sizeof(p));
	p.alm = s->d_alm; p.almoff = s->d_almoff;
	p.lmax = s->lmax; p.mmax = s->mmax; p.mres = s->mres;
	p.ltr = s->lmax; p.mtr = s->mmax;
	return p;
}

size_t al16(size_t b) { return (b + 255) & ~(size_t) 255; }

// host spectra -> device staging; returns the device pointers (null where the host pointer is null)
bool stage_spectra(shtns_cfg s, long n, const cplx* const* in, int nin, size_t extra, double2** dev, char** rest)
{
	const size_t sb = al16(sizeof(double2) * (size_t) n);
	char* base = static_cast<char*>(loc_buf(s, nin * sb + extra));
	if (!base) return false;
	for (int i = 0; i < nin; i++) {
		dev[i] = nullptr;
		if (in[i]) {
			dev[i] = reinterpret_cast<double2*>(base + i * sb);
			cudaMemcpyAsync(dev[i], in[i], sizeof(double2) * n, cudaMemcpyHostToDevice, s->comp_stream);
		}
	}
	*rest = base + nin * sb;
	return true;
}

bool loc_check(shtns_cfg s)
{
	if (!s) { shtb_set_error(1, "local evaluation on a null plan"); return false; }
	return loc_tables(s);
}

// point evaluation of real fields (Q, S, T host pointers; ncomp 1 or 3)
void point_host(shtns_cfg s, const cplx* Q, const cplx* S, const cplx* T, double cost, double phi, int ncomp,
                double* vr, double* vt, double* vp)
{
	if (!loc_check(s)) return;
	const cplx* in[3] = {Q, S, T};
	double2* d[3];
	char* rest;
	if (!stage_spectra(s, s->nlm, in, 3, 256, d, &rest)) return;
	double* buf = reinterpret_cast<double*>(rest);          // cost, phi, v0, v1, v2
	double hb[2] = {cost, phi};
	cudaMemcpyAsync(buf, hb, sizeof(hb), cudaMemcpyHostToDevice, s->comp_stream);
	LocalParams p = loc_params(s);
	p.Q = d[0]; p.S = d[1]; p.T = d[2];
	point_kernel<<<1, PT_THREADS, 0, s->comp_stream>>>(p, buf, buf + 1, ncomp, 0, buf + 2, buf + 3, buf + 4);
	shtb_count_launch();
	if (!shtb_cuda_ok(cudaGetLastError(), "point evaluation launch")) return;
	double out[3] = {0.0, 0.0, 0.0};
	cudaMemcpyAsync(out, buf + 2, sizeof(out), cudaMemcpyDeviceToHost, s->comp_stream);
	if (!shtb_cuda_ok(cudaStreamSynchronize(s->comp_stream), "point evaluation")) return;
	if (vr) *vr = out[0];
	if (vt) *vt = out[1];
	if (vp) *vp = out[2];
}

void lat_host(shtns_cfg s, const cplx* Q, const cplx* S, const cplx* T, double cost, int ncomp,
              double* vr, double* vt, double* vp, int nphi, int ltr, int mtr)
{
	if (!loc_check(s)) return;
	if (nphi <= 0) { shtb_set_error(1, "SH_to_lat: nphi must be positive"); return; }
	// truncation as the reference (sht_func.c:741-744)
	if (ltr > s->lmax) ltr = s->lmax;
	if (ltr < 0) ltr = 0;
	if (mtr > s->mmax) mtr = s->mmax;
	if (mtr * s->mres > ltr) mtr = ltr / s->mres;
	if (mtr * 2 * s->mres >= nphi) mtr = (nphi - 1) / (2 * s->mres);
	if (mtr < 0) mtr = 0;
	const int nm = mtr + 1;
	const cplx* in[3] = {Q, S, T};
	double2* d[3];
	char* rest;
	const size_t fb = al16(sizeof(double2) * 3 * nm), vb = sizeof(double) * 3 * (size_t) nphi;
	if (!stage_spectra(s, s->nlm, in, 3, fb + vb, d, &rest)) return;
	double2* F = reinterpret_cast<double2*>(rest);
	double* v = reinterpret_cast<double*>(rest + fb);
	LocalParams p = loc_params(s);
	p.Q = d[0]; p.S = d[1]; p.T = d[2];
	p.ltr = ltr; p.mtr = mtr; p.F = F; p.nm = nm;
	const double st = sqrt((1.0 - cost) * (1.0 + cost));
	lat_coef_kernel<<<(nm + 127) / 128, 128, 0, s->comp_stream>>>(p, cost, st);
	lat_dft_kernel<<<(nphi + 127) / 128, 128, 0, s->comp_stream>>>(F, nm, s->mres, nphi, ncomp, v, v + nphi, v + 2 * nphi);
	shtb_count_launch(2);
	if (!shtb_cuda_ok(cudaGetLastError(), "latitude evaluation launch")) return;
	double* outs[3] = {vr, vt, vp};
	for (int c = 0; c < ncomp; c++)
		cudaMemcpyAsync(outs[c], v + (size_t) c * nphi, sizeof(double) * nphi, cudaMemcpyDeviceToHost, s->comp_stream);
	shtb_cuda_ok(cudaStreamSynchronize(s->comp_stream), "latitude evaluation");
}

int legendre_host(shtns_cfg s, int lmax, int im, double x, double sint, double* yl, double* dyl, int deriv)
{
	if (!loc_check(s)) return 0;
	if (im < 0 || im > s->mmax || lmax < im * s->mres || lmax > s->lmax + 1) {
		shtb_set_error(1, "legendre_sphPlm_array: argument out of range");
		return 0;
	}
	const int m = im * s->mres, n = lmax - m + 1;
	char* base = static_cast<char*>(loc_buf(s, sizeof(double) * 2 * (size_t) n + 64));
	if (!base) return 0;
	double* y = reinterpret_cast<double*>(base);
	double* dy = y + n;
	int* lnz = reinterpret_cast<int*>(dy + n);
	LocalParams p = loc_params(s);
	p.ltr = lmax; p.yl = y; p.dyl = deriv ? dy : nullptr; p.lnz = lnz;
	legendre_array_kernel<<<1, 32, 0, s->comp_stream>>>(p, im, x, sint, deriv);
	shtb_count_launch();
	if (!shtb_cuda_ok(cudaGetLastError(), "Legendre array launch")) return 0;
	int first = 0;
	cudaMemcpyAsync(yl, y, sizeof(double) * n, cudaMemcpyDeviceToHost, s->comp_stream);
	if (deriv) cudaMemcpyAsync(dyl, dy, sizeof(double) * n, cudaMemcpyDeviceToHost, s->comp_stream);
	cudaMemcpyAsync(&first, lnz, sizeof(int), cudaMemcpyDeviceToHost, s->comp_stream);
	if (!shtb_cuda_ok(cudaStreamSynchronize(s->comp_stream), "Legendre array")) return 0;
	return first;
}

} // namespace

// Legendre values of all orders of plan s (mres = 1) at x = cos(theta), for
// the rotation tables (enqueued on stream st_)
void launch_plm_table(shtns_cfg s, double x, double st, double* out, cudaStream_t st_)
{
	if (!loc_check(s)) return;
	LocalParams p = loc_params(s);
	plm_table_kernel<<<(s->mmax + 1 + 127) / 128, 128, 0, st_>>>(p, x, st, out);
	shtb_count_launch();
	shtb_cuda_ok(cudaGetLastError(), "Legendre table launch");
}

// ---- points (sht_func.c:516-730) ----
extern "C" double SH_to_point(shtns_cfg s, cplx* Qlm, double cost, double phi)
{
	double v = 0.0;
	point_host(s, Qlm, nullptr, nullptr, cost, phi, 1, &v, nullptr, nullptr);
	return v;
}

extern "C" void SHqst_to_point(shtns_cfg s, cplx* Qlm, cplx* Slm, cplx* Tlm, double cost, double phi,
                               double* vr, double* vt, double* vp)
{
	point_host(s, Qlm, Slm, Tlm, cost, phi, 3, vr, vt, vp);
}

extern "C" void SH_to_grad_point(shtns_cfg s, cplx* DrSlm, cplx* Slm, double cost, double phi,
                                 double* vr, double* vt, double* vp)
{
	point_host(s, DrSlm, Slm, nullptr, cost, phi, 3, vr, vt, vp);
}

extern "C" cplx SH_to_point_cplx(shtns_cfg s, cplx* alm, double cost, double phi)
{
	double out[2] = {0.0, 0.0};
	cplx z;
	memset(&z, 0, sizeof(z));
	if (!loc_check(s)) return z;
	if (s->mres != 1) { shtb_set_error(1, "SH_to_point_cplx: mres must be 1"); return z; }
	const cplx* in[1] = {alm};
	double2* d[1];
	char* rest;
	if (!stage_spectra(s, s->nlm_cplx, in, 1, 256, d, &rest)) return z;
	double* buf = reinterpret_cast<double*>(rest);
	double hb[2] = {cost, phi};
	cudaMemcpyAsync(buf, hb, sizeof(hb), cudaMemcpyHostToDevice, s->comp_stream);
	LocalParams p = loc_params(s);
	p.Q = d[0]; p.cplx = 1;
	point_kernel<<<1, PT_THREADS, 0, s->comp_stream>>>(p, buf, buf + 1, 1, 1, buf + 2, nullptr, nullptr);
	shtb_count_launch();
	if (!shtb_cuda_ok(cudaGetLastError(), "point evaluation launch")) return z;
	cudaMemcpyAsync(out, buf + 2, sizeof(out), cudaMemcpyDeviceToHost, s->comp_stream);
	if (!shtb_cuda_ok(cudaStreamSynchronize(s->comp_stream), "point evaluation")) return z;
	memcpy(&z, out, sizeof(out));
	return z;
}

// ---- one latitude (sht_func.c:732-885) ----
extern "C" void SH_to_lat(shtns_cfg s, cplx* Qlm, double cost, double* vr, int nphi, int ltr, int mtr)
{
	lat_host(s, Qlm, nullptr, nullptr, cost, 1, vr, nullptr, nullptr, nphi, ltr, mtr);
}

extern "C" void SHqst_to_lat(shtns_cfg s, cplx* Qlm, cplx* Slm, cplx* Tlm, double cost,
                             double* vr, double* vt, double* vp, int nphi, int ltr, int mtr)
{
	lat_host(s, Qlm, Slm, Tlm, cost, 3, vr, vt, vp, nphi, ltr, mtr);
}

// ---- Legendre arrays (sht_legendre.c:238-440) ----
extern "C" int legendre_sphPlm_array(shtns_cfg s, const int lmax, const int im, const double x, double* yl)
{
	return legendre_host(s, lmax, im, x, sqrt((1.0 - x) * (1.0 + x)), yl, nullptr, 0);
}

extern "C" int legendre_sphPlm_deriv_array(shtns_cfg s, const int lmax, const int im, const double x, const double sint,
                                           double* yl, double* dyl)
{
	return legendre_host(s, lmax, im, x, sint, yl, dyl, 1);
}

// ---- l+-1 operators (sht_func.c:484-507) ----
extern "C" void SH_mul_mx(shtns_cfg s, double* mx, cplx* Qlm, cplx* Rlm)
{
	if (!s || !mx || !Qlm || !Rlm) { shtb_set_error(1, "SH_mul_mx: null argument"); return; }
	const long n = s->nlm;
	const size_t qb = al16(sizeof(double2) * n), mb = al16(sizeof(double) * 2 * n);
	char* base = static_cast<char*>(loc_buf(s, 2 * qb + mb));
	if (!base) return;
	double2* q = reinterpret_cast<double2*>(base);
	double2* r = reinterpret_cast<double2*>(base + qb);
	double* m = reinterpret_cast<double*>(base + 2 * qb);
	cudaMemcpyAsync(q, Qlm, sizeof(double2) * n, cudaMemcpyHostToDevice, s->comp_stream);
	cudaMemcpyAsync(m, mx, sizeof(double) * 2 * n, cudaMemcpyHostToDevice, s->comp_stream);
	mul_mx_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s->comp_stream>>>(m, q, r, n);
	shtb_count_launch();
	if (!shtb_cuda_ok(cudaGetLastError(), "SH_mul_mx launch")) return;
	cudaMemcpyAsync(Rlm, r, sizeof(double2) * n, cudaMemcpyDeviceToHost, s->comp_stream);
	shtb_cuda_ok(cudaStreamSynchronize(s->comp_stream), "SH_mul_mx");
}

// ---- batched device forms (no counterpart in the reference) ----
extern "C" void shtns_b200_SH_to_points(shtns_cfg s, cplx* Qlm, const double* cost, const double* phi, double* v, int npts)
{
	if (!loc_check(s) || npts <= 0) return;
	LocalParams p = loc_params(s);
	p.Q = reinterpret_cast<const double2*>(Qlm);
	point_kernel<<<npts, PT_THREADS, 0, s->comp_stream>>>(p, cost, phi, 1, 0, v, nullptr, nullptr);
	shtb_count_launch();
	shtb_cuda_ok(cudaGetLastError(), "point evaluation launch");
}

extern "C" void shtns_b200_SHqst_to_points(shtns_cfg s, cplx* Qlm, cplx* Slm, cplx* Tlm, const double* cost,
                                           const double* phi, double* vr, double* vt, double* vp, int npts)
{
	if (!loc_check(s) || npts <= 0) return;
	LocalParams p = loc_params(s);
	p.Q = reinterpret_cast<const double2*>(Qlm);
	p.S = reinterpret_cast<const double2*>(Slm);
	p.T = reinterpret_cast<const double2*>(Tlm);
	point_kernel<<<npts, PT_THREADS, 0, s->comp_stream>>>(p, cost, phi, 3, 0, vr, vt, vp);
	shtb_count_launch();
	shtb_cuda_ok(cudaGetLastError(), "point evaluation launch");
}
