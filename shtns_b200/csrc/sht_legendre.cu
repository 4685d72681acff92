// Legendre stage of the spherical-harmonic transforms on sm_100a.
//
// Per azimuthal order m the Legendre sum is a real matrix product with an
// on-the-fly left operand:
//   synthesis  E/O[theta, col] = sum_k Y_k(theta) * qq[k, col]
//   analysis   qq[k, col]      = sum_theta Y_k(theta) * G[theta, col]
// where Y_k(theta) = sin^m(theta) * p_k(cos^2 theta) follows Ishioka's two-term
// recurrence Y_{k+1} = (c_{2k+1} x^2 + c_{2k}) Y_k + Y_{k-1} (the reference's
// SHT/kernel_SH_to_spat.gen.c:388-409 and kernel_spat_to_SH.gen.c:541-598),
// `col` runs over field-components x {even, odd} x {re, im}, and the even
// and odd degrees share Y_k (the odd part is multiplied by cos(theta) when the
// hemispheres are folded, kernel_SH_to_spat.gen.c:429-441).
//
// The product runs on the FP64 tensor cores (mma.sync m8n8k4 f64: tcgen05 has
// no FP64 kind).  Each CTA regenerates its Y tile in shared memory from
// recurrence checkpoints (Y_k, Y_{k+1}) stored every 32 degrees, so tiles can
// start at any k and the recurrence of one tile is only 32 dependent steps.
#include "sht_internal.h"

namespace {

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b)
{
	asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
	             : "+d"(c[0]), "+d"(c[1]) : "d"(a), "d"(b));
}

// ---------------------------------------------------------------------------
// Checkpoints: thread (t, im) runs the recurrence of order m at north row t and
// stores (Y_{32s}, Y_{32s+1}) for every segment s.  Y_0 = sin^m(theta) by
// binary powering (sint_pow_n_ext, sht_legendre.c:110-139, without the range
// extension: below lmax 1800 an underflowed seed only drops values below
// 1e-300), Y_1 = (c_1 x^2 + c_0) Y_0 (kernel_SH_to_spat.gen.c:303-315).
__global__ void ck_kernel(int nlat_2, int mres, const double* __restrict__ x2g, const double* __restrict__ sing,
                          const double* __restrict__ c, MTables mt, const int* __restrict__ nseg, double2* __restrict__ ck)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	const int im = blockIdx.y;
	if (t >= nlat_2) return;
	const int m = im * mres;
	const double x2 = x2g[t];
	double y0 = 1.0, b = sing[t];
	for (int n = m; n; n >>= 1) {
		if (n & 1) y0 *= b;
		b *= b;
	}
	const double* cc = c + mt.coff[im];
	double y1 = fma(cc[1], x2, cc[0]) * y0;
	const int ns = nseg[im];
	double2* out = ck + (long)mt.ckoff[im] * nlat_2 + t;
	for (int s = 0; s < ns; s++) {
		out[(long)s * nlat_2] = make_double2(y0, y1);
		const int kb = s * LG_SEG + 1;
		#pragma unroll 4
		for (int j = 0; j < LG_SEG; j++) {
			const int k = kb + j;
			const double a = fma(cc[2 * k + 1], x2, cc[2 * k]);
			const double y2 = fma(a, y1, y0);
			y0 = y1;
			y1 = y2;
		}
	}
}

// ---------------------------------------------------------------------------
// Synthesis prologue: spectral coefficients -> Ishioka basis, k-major layout.
//   even: qe_k = X0_k Q_{m+2k} + X1_k Q_{m+2k+2};  odd: qo_k = X2_k Q_{m+2k+1}
// (SH_to_ishioka, sht_private.h:442-483).  Vector components first form
//   V_l =  (st d/dth S)_l + i m T_l,  W_l = -(st d/dth T)_l + i m S_l
// for l = m..llim+1 (SH_vect_to_2scal, sht_private.h:534-584).
// Column layout: field-component fc owns columns 16*(fc/4) + 2*(fc%4) + {0,1}
// (even re, im) and the same +8 (odd re, im).
__device__ __forceinline__ double2 ld_coef(const double2* base, long off, int j, int lrel_max, bool m0)
{
	if (base == nullptr || j < 0 || j > lrel_max) return make_double2(0.0, 0.0);
	double2 v = base[off + j];
	if (m0) v.y = 0.0;
	return v;
}

__device__ __forceinline__ double2 vw_coef(const PrepParams& p, int type, long off, int f, int m, int voff,
                                           int j, int lrel_max, bool m0)
{
	// degree l = m + j, valid up to llim + 1 (lrel_max + 1)
	if (j < 0 || j > lrel_max + 1) return make_double2(0.0, 0.0);
	const double lo = (j > 0) ? p.stdt_lo[voff + j] : 0.0;
	const double hi = p.stdt_hi[voff + j];
	const long o = off + (long)f * p.spec_dist;
	const double2 sm = ld_coef(p.S, o, j - 1, lrel_max, m0), sp = ld_coef(p.S, o, j + 1, lrel_max, m0);
	const double2 tmm = ld_coef(p.T, o, j - 1, lrel_max, m0), tp = ld_coef(p.T, o, j + 1, lrel_max, m0);
	const double2 s0 = ld_coef(p.S, o, j, lrel_max, m0), t0 = ld_coef(p.T, o, j, lrel_max, m0);
	const double em = (double)m;
	if (type == 1) {   // V = stdt S + i m T
		return make_double2(lo * sm.x + hi * sp.x - em * t0.y, lo * sm.y + hi * sp.y + em * t0.x);
	} else {           // W = -stdt T + i m S
		return make_double2(-(lo * tmm.x + hi * tp.x) - em * s0.y, -(lo * tmm.y + hi * tp.y) + em * s0.x);
	}
}

__global__ void prep_synth_kernel(PrepParams p)
{
	const int im = blockIdx.y;
	if (im > p.mlim) return;
	const int m = im * p.mres;
	const int nfc = p.nf * p.ncomp;
	const int kmax = (p.llim + 1 - m) / 2 + 1;
	const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= (long)kmax * nfc) return;
	const int k = (int)(idx / nfc);
	const int fc = (int)(idx - (long)k * nfc);
	const int comp = fc / p.nf, f = fc - comp * p.nf;
	const int type = p.comp_type[comp];
	const bool m0 = (m == 0);
	const int lrel_max = p.llim - m;
	const long off = (long)im * (2 * p.lmax + 2 - (im + 1) * p.mres) / 2 + m;   // LM(m, m)
	const double* X = p.xs + p.mt.xoff[im] + 3 * k;
	double2 qa, qb, qc;   // relative degrees 2k, 2k+1, 2k+2
	if (type == 0) {
		const double2* Q = p.Q;
		const long o = off + (long)f * p.spec_dist;
		qa = ld_coef(Q, o, 2 * k, lrel_max, m0);
		qb = ld_coef(Q, o, 2 * k + 1, lrel_max, m0);
		qc = ld_coef(Q, o, 2 * k + 2, lrel_max, m0);
	} else {
		const int voff = p.mt.voff[im];
		qa = vw_coef(p, type, off, f, m, voff, 2 * k, lrel_max, m0);
		qb = vw_coef(p, type, off, f, m, voff, 2 * k + 1, lrel_max, m0);
		qc = vw_coef(p, type, off, f, m, voff, 2 * k + 2, lrel_max, m0);
	}
	const double x0 = X[0], x1 = X[1], x2 = X[2];
	const double2 qe = make_double2(fma(x0, qa.x, x1 * qc.x), fma(x0, qa.y, x1 * qc.y));
	const double2 qo = make_double2(x2 * qb.x, x2 * qb.y);
	double* row = p.qq + (long)(p.mt.koff[im] + k) * p.ncol;
	const int ce = 16 * (fc >> 2) + 2 * (fc & 3);
	*reinterpret_cast<double2*>(row + ce) = qe;
	*reinterpret_cast<double2*>(row + ce + 8) = qo;
}

// ---------------------------------------------------------------------------
// Analysis epilogue: Ishioka basis -> spectral coefficients
//   Q_{m+2k} = X0_k e_k + X1_{k-1} e_{k-1},  Q_{m+2k+1} = X2_k o_k
// (ishioka_to_SH, sht_private.h:345-374), and for vectors
//   S_l = -((MX V)_l + i m W_l) / (l(l+1)),  T_l = -(i m V_l - (MX W)_l) / (l(l+1))
// with MX = 2 cos + sin d/dtheta (SH_2scal_to_vect, sht_private.h:296-337).
// Degrees above llim and orders above mlim are written as zero (SHT_VAR_LTR).
__device__ __forceinline__ double2 ish_inv(const PrepParams& p, const double* X, long row0, int col, int j)
{
	if (j < 0) return make_double2(0.0, 0.0);
	const int k = j >> 1;
	if ((j & 1) == 0) {
		const double2 e = *reinterpret_cast<const double2*>(p.qq + (row0 + k) * p.ncol + col);
		double2 r = make_double2(X[3 * k] * e.x, X[3 * k] * e.y);
		if (k > 0) {
			const double2 e1 = *reinterpret_cast<const double2*>(p.qq + (row0 + k - 1) * p.ncol + col);
			r.x = fma(X[3 * (k - 1) + 1], e1.x, r.x);
			r.y = fma(X[3 * (k - 1) + 1], e1.y, r.y);
		}
		return r;
	} else {
		const double2 o = *reinterpret_cast<const double2*>(p.qq + (row0 + k) * p.ncol + col + 8);
		return make_double2(X[3 * k + 2] * o.x, X[3 * k + 2] * o.y);
	}
}

__global__ void post_analys_kernel(PrepParams p)
{
	// one thread per (degree, field, output group); group 0 = scalar Q (if any),
	// group g>0 = vector pair (S, T)
	const int im = blockIdx.y;
	const int m = im * p.mres;
	const int nl = p.lmax - m + 1;
	const int ngroups = (p.comp_type[0] == 0) ? 1 + (p.ncomp > 1 ? 1 : 0) : 1;
	const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= (long)nl * p.nf * ngroups) return;
	const int j = (int)(idx % nl);
	const int rest = (int)(idx / nl);
	const int f = rest % p.nf;
	const int g = rest / p.nf;
	const long off = (long)im * (2 * p.lmax + 2 - (im + 1) * p.mres) / 2 + m;
	const long o = off + (long)f * p.spec_dist + j;
	const int l = m + j;
	const bool scalar_group = (p.comp_type[0] == 0) && (g == 0);
	const bool zero = (im > p.mlim) || (l > p.llim);
	if (scalar_group) {
		double2 q = make_double2(0.0, 0.0);
		if (!zero) {
			const int fc = f;   // scalar component is component 0
			const int ce = 16 * (fc >> 2) + 2 * (fc & 3);
			q = ish_inv(p, p.xa + p.mt.xoff[im], p.mt.koff[im], ce, j);
			if (m == 0) q.y = 0.0;
		}
		p.Qo[o] = q;
		return;
	}
	// vector pair: components V (type 1) and W (type 2)
	const int cv = (p.comp_type[0] == 0) ? 1 : 0;
	double2 s = make_double2(0.0, 0.0), t = make_double2(0.0, 0.0);
	if (!zero) {
		const int fcv = cv * p.nf + f, fcw = (cv + 1) * p.nf + f;
		const int cev = 16 * (fcv >> 2) + 2 * (fcv & 3);
		const int cew = 16 * (fcw >> 2) + 2 * (fcw & 3);
		const double* X = p.xa + p.mt.xoff[im];
		const long r0 = p.mt.koff[im];
		const double2 vm = ish_inv(p, X, r0, cev, j - 1), v0 = ish_inv(p, X, r0, cev, j), vp = ish_inv(p, X, r0, cev, j + 1);
		const double2 wm = ish_inv(p, X, r0, cew, j - 1), w0 = ish_inv(p, X, r0, cew, j), wp = ish_inv(p, X, r0, cew, j + 1);
		const int voff = p.mt.voff[im];
		const double lo = (j > 0) ? p.van_lo[voff + j] : 0.0;
		const double hi = p.van_hi[voff + j];
		const double l2 = p.l2[l];
		const double em = (double)m;
		const double mxv_r = lo * vm.x + hi * vp.x, mxv_i = lo * vm.y + hi * vp.y;
		const double mxw_r = lo * wm.x + hi * wp.x, mxw_i = lo * wm.y + hi * wp.y;
		// i m W = (-m W.y, m W.x)
		s = make_double2(-(mxv_r - em * w0.y) * l2, -(mxv_i + em * w0.x) * l2);
		t = make_double2(-(-em * v0.y - mxw_r) * l2, -(em * v0.x - mxw_i) * l2);
		if (m == 0) { s.y = 0.0; t.y = 0.0; }
	}
	p.So[o] = s;
	p.To[o] = t;
}

// ---------------------------------------------------------------------------
// Synthesis contraction.  CTA = (order im, 64 north theta rows, 64 columns).
// 8 warps as 2 (theta) x 4 (columns); a warp owns 32 rows x 16 columns = one
// group of 4 field-components, so each lane ends with (E_re, E_im, O_re, O_im)
// of one (row, field-component) and folds north/south itself.
#define SA_LD 68   // shared row stride in doubles: 4 mod 16 keeps fragment loads conflict-free

__global__ void __launch_bounds__(LG_THREADS)
leg_synth_kernel(LegParams p)
{
	__shared__ __align__(16) double As[LG_BK][SA_LD];   // [k][theta]
	__shared__ __align__(16) double Bs[LG_BK][SA_LD];   // [k][col]
	const int im = blockIdx.y;
	const int m = im * p.mres;
	const int ntb = (p.nlat_2 + LG_BM - 1) / LG_BM;
	const int tb = blockIdx.x % ntb, nb = blockIdx.x / ntb;
	const int t0 = tb * LG_BM, c0 = nb * LG_BN;
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int wm = warp >> 2, wn = warp & 3;
	const int nk = (p.llim + p.vec_extra - m) / 2 + 1;
	const int tmm = p.mt.tm[im];

	double acc[4][2][2];
	#pragma unroll
	for (int i = 0; i < 4; i++)
		#pragma unroll
		for (int j = 0; j < 2; j++) { acc[i][j][0] = 0.0; acc[i][j][1] = 0.0; }

	if (t0 + LG_BM > tmm) {
		const double* cm = p.c + p.mt.coff[im];
		const double2* ckm = p.ck + (long)p.mt.ckoff[im] * p.nlat_2;
		const double* qrow = p.qq + (long)p.mt.koff[im] * p.ncol;
		for (int k0 = 0; k0 < nk; k0 += LG_BK) {
			if (tid < LG_BM) {
				const int t = t0 + tid;
				double y0 = 0.0, y1 = 0.0, x2 = 0.0;
				if (t < p.nlat_2) {
					const double2 s = ckm[(long)(k0 / LG_SEG) * p.nlat_2 + t];
					y0 = s.x; y1 = s.y; x2 = p.x2[t];
				}
				As[0][tid] = y0;
				As[1][tid] = y1;
				const double* cc = cm + 2 * k0;
				#pragma unroll 6
				for (int j = 2; j < LG_BK; j++) {
					const double a = fma(cc[2 * j - 1], x2, cc[2 * j - 2]);
					const double y2 = fma(a, y1, y0);
					As[j][tid] = y2;
					y0 = y1; y1 = y2;
				}
			}
			for (int e = tid; e < LG_BK * (LG_BN / 2); e += LG_THREADS) {
				const int kk = e / (LG_BN / 2), cc2 = (e - kk * (LG_BN / 2)) * 2;
				const int k = k0 + kk, col = c0 + cc2;
				double2 v = make_double2(0.0, 0.0);
				if (k < nk && col < p.ncol) v = *reinterpret_cast<const double2*>(qrow + (long)k * p.ncol + col);
				Bs[kk][cc2] = v.x;
				Bs[kk][cc2 + 1] = v.y;
			}
			__syncthreads();
			#pragma unroll
			for (int kk = 0; kk < LG_BK; kk += 4) {
				double a[4], b[2];
				#pragma unroll
				for (int i = 0; i < 4; i++) a[i] = As[kk + (lane & 3)][wm * 32 + i * 8 + (lane >> 2)];
				#pragma unroll
				for (int j = 0; j < 2; j++) b[j] = Bs[kk + (lane & 3)][wn * 16 + j * 8 + (lane >> 2)];
				#pragma unroll
				for (int i = 0; i < 4; i++)
					#pragma unroll
					for (int j = 0; j < 2; j++) dmma(acc[i][j], a[i], b[j]);
			}
			__syncthreads();
		}
	}
	// epilogue: fold hemispheres, apply 1/sin for vector components, store F
	const int fc = ((c0 + wn * 16) >> 4) * 4 + (lane & 3);
	if (fc >= p.nfc) return;
	const bool vec = (p.ctype[fc / p.nf] != 0) && !p.robert;
	double2* Ff = p.F + (long)fc * p.fstride + (long)im * p.nlat;
	#pragma unroll
	for (int i = 0; i < 4; i++) {
		const int t = t0 + wm * 32 + i * 8 + (lane >> 2);
		if (t >= p.nlat_2) continue;
		const double cx = p.x[t];
		double nr = fma(cx, acc[i][1][0], acc[i][0][0]), ni = fma(cx, acc[i][1][1], acc[i][0][1]);
		double sr = fma(-cx, acc[i][1][0], acc[i][0][0]), si = fma(-cx, acc[i][1][1], acc[i][0][1]);
		if (t < tmm) { nr = ni = sr = si = 0.0; }
		if (vec) { const double s = p.sinv[t]; nr *= s; ni *= s; sr *= s; si *= s; }
		const int rn = p.south_first ? p.nlat - 1 - t : t;
		const int rs = p.nlat - 1 - rn;
		Ff[rn] = make_double2(nr, ni);
		Ff[rs] = make_double2(sr, si);
	}
}

// ---------------------------------------------------------------------------
// Analysis contraction.  CTA = (order im, 64 k rows, 64 columns); the K loop
// runs over north theta rows in chunks of 32, starting at the polar threshold.
// The B operand is built while staging: G_even = w (F_N + F_S),
// G_odd = w cos(theta) (F_N - F_S) (kernel_spat_to_SH.gen.c:485-491), times
// 1/sin(theta) for vector components (1/sin^2 in Robert form).
#define AA_LD 36   // As row stride (k rows x 32 theta): 4 mod 16

__global__ void __launch_bounds__(LG_THREADS)
leg_analys_kernel(LegParams p, int nkb)
{
	__shared__ __align__(16) double As[LG_BM][AA_LD];   // [k][theta]
	__shared__ __align__(16) double Bs[LG_BK][SA_LD];   // [theta][col]
	const int im = blockIdx.y;
	const int m = im * p.mres;
	const int kb = blockIdx.x % nkb, nb = blockIdx.x / nkb;
	const int k0 = kb * LG_BM, c0 = nb * LG_BN;
	const int nk = (p.llim + p.vec_extra - m) / 2 + 1;
	if (k0 >= nk) return;
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int wm = warp >> 2, wn = warp & 3;
	const int tmm = p.mt.tm[im];
	const double wfac = (m > 0) ? p.mpos_inv : 1.0;
	const double* cm = p.c + p.mt.coff[im];
	const double2* ckm = p.ck + (long)p.mt.ckoff[im] * p.nlat_2;
	const int fc0 = c0 / 4;

	double acc[4][2][2];
	#pragma unroll
	for (int i = 0; i < 4; i++)
		#pragma unroll
		for (int j = 0; j < 2; j++) { acc[i][j][0] = 0.0; acc[i][j][1] = 0.0; }

	for (int tt0 = (tmm / LG_BK) * LG_BK; tt0 < p.nlat_2; tt0 += LG_BK) {
		if (tid < 2 * LG_BK) {
			const int tt = tid & (LG_BK - 1), sgi = tid / LG_BK;
			const int t = tt0 + tt, ks = k0 + sgi * LG_SEG;
			double y0 = 0.0, y1 = 0.0, x2 = 0.0;
			if (t < p.nlat_2 && ks < nk) {
				const double2 s = ckm[(long)(ks / LG_SEG) * p.nlat_2 + t];
				y0 = s.x; y1 = s.y; x2 = p.x2[t];
			}
			double* a = &As[sgi * LG_SEG][tt];
			a[0] = y0;
			a[AA_LD] = y1;
			if (ks < nk) {
				const double* cc = cm + 2 * ks;
				#pragma unroll 6
				for (int j = 2; j < LG_SEG; j++) {
					const double aa = fma(cc[2 * j - 1], x2, cc[2 * j - 2]);
					const double y2 = fma(aa, y1, y0);
					a[j * AA_LD] = y2;
					y0 = y1; y1 = y2;
				}
			} else {
				for (int j = 2; j < LG_SEG; j++) a[j * AA_LD] = 0.0;
			}
		}
		for (int e = tid; e < LG_BK * (LG_BN / 4); e += LG_THREADS) {
			const int tt = e % LG_BK, fl = e / LG_BK;
			const int t = tt0 + tt, fc = fc0 + fl;
			double er = 0.0, ei = 0.0, orr = 0.0, oi = 0.0;
			if (t < p.nlat_2 && t >= tmm && fc < p.nfc) {
				const int rn = p.south_first ? p.nlat - 1 - t : t;
				const int rs = p.nlat - 1 - rn;
				const double2* Ff = p.F + (long)fc * p.fstride + (long)im * p.nlat;
				const double2 fn = Ff[rn], fs = Ff[rs];
				double w = p.w[t] * wfac;
				if (p.ctype[fc / p.nf] != 0) {
					double s = p.sinv[t];
					if (p.robert) s *= s;
					w *= s;
				}
				const double wo = w * p.x[t];
				er = w * (fn.x + fs.x);  ei = w * (fn.y + fs.y);
				orr = wo * (fn.x - fs.x); oi = wo * (fn.y - fs.y);
			}
			const int cb = 16 * (fl >> 2) + 2 * (fl & 3);
			Bs[tt][cb] = er;  Bs[tt][cb + 1] = ei;
			Bs[tt][cb + 8] = orr;  Bs[tt][cb + 9] = oi;
		}
		__syncthreads();
		#pragma unroll
		for (int kk = 0; kk < LG_BK; kk += 4) {
			double a[4], b[2];
			#pragma unroll
			for (int i = 0; i < 4; i++) a[i] = As[wm * 32 + i * 8 + (lane >> 2)][kk + (lane & 3)];
			#pragma unroll
			for (int j = 0; j < 2; j++) b[j] = Bs[kk + (lane & 3)][wn * 16 + j * 8 + (lane >> 2)];
			#pragma unroll
			for (int i = 0; i < 4; i++)
				#pragma unroll
				for (int j = 0; j < 2; j++) dmma(acc[i][j], a[i], b[j]);
		}
		__syncthreads();
	}
	double* qrow = p.qq + (long)p.mt.koff[im] * p.ncol;
	#pragma unroll
	for (int i = 0; i < 4; i++) {
		const int k = k0 + wm * 32 + i * 8 + (lane >> 2);
		if (k >= nk) continue;
		#pragma unroll
		for (int j = 0; j < 2; j++) {
			const int col = c0 + wn * 16 + j * 8 + (lane & 3) * 2;
			if (col < p.ncol)
				*reinterpret_cast<double2*>(qrow + (long)k * p.ncol + col) = make_double2(acc[i][j][0], acc[i][j][1]);
		}
	}
}

} // namespace

// ---------------------------------------------------------------------------
void launch_checkpoints(shtns_cfg s, cudaStream_t st)
{
	std::vector<int> nseg(s->mmax + 1);
	for (int im = 0; im <= s->mmax; im++) nseg[im] = (s->kmax_h[im] + LG_SEG - 1) / LG_SEG;
	int* d_nseg = nullptr;
	if (!shtb_cuda_ok(cudaMalloc(&d_nseg, sizeof(int) * nseg.size()), "checkpoint table")) return;
	cudaMemcpyAsync(d_nseg, nseg.data(), sizeof(int) * nseg.size(), cudaMemcpyHostToDevice, st);
	dim3 grid((s->nlat_2 + 127) / 128, s->mmax + 1);
	ck_kernel<<<grid, 128, 0, st>>>(s->nlat_2, s->mres, s->d_x2, s->d_s, s->d_c, s->mt, d_nseg, s->d_ck);
	shtb_count_launch();
	shtb_cuda_ok(cudaGetLastError(), "checkpoint kernel");
	cudaStreamSynchronize(st);
	cudaFree(d_nseg);
}

void launch_prep_synth(const PrepParams& p, cudaStream_t st)
{
	const int nfc = p.nf * p.ncomp;
	const long rows = (long)((p.llim + 1) / 2 + 1) * nfc;
	dim3 grid((unsigned)((rows + 255) / 256), p.mlim + 1);
	prep_synth_kernel<<<grid, 256, 0, st>>>(p);
	shtb_count_launch();
}

void launch_leg_synth(const LegParams& p, cudaStream_t st)
{
	const int ntb = (p.nlat_2 + LG_BM - 1) / LG_BM;
	const int nnb = (p.ncol + LG_BN - 1) / LG_BN;
	dim3 grid(ntb * nnb, p.mlim + 1);
	leg_synth_kernel<<<grid, LG_THREADS, 0, st>>>(p);
	shtb_count_launch();
}

void launch_leg_analys(const LegParams& p, int kmax_all, cudaStream_t st)
{
	const int nkb = (kmax_all + LG_BM - 1) / LG_BM;
	const int nnb = (p.ncol + LG_BN - 1) / LG_BN;
	dim3 grid(nkb * nnb, p.mlim + 1);
	leg_analys_kernel<<<grid, LG_THREADS, 0, st>>>(p, nkb);
	shtb_count_launch();
}

void launch_post_analys_m(const PrepParams& p, int mmax, cudaStream_t st)
{
	const int ngroups = (p.comp_type[0] == 0) ? 1 + (p.ncomp > 1 ? 1 : 0) : 1;
	const long n = (long)(p.lmax + 1) * p.nf * ngroups;
	dim3 grid((unsigned)((n + 255) / 256), mmax + 1);
	post_analys_kernel<<<grid, 256, 0, st>>>(p);
	shtb_count_launch();
}
