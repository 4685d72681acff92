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
// The product runs on the FP64 tensor cores (mma.sync m16n8k4 f64: tcgen05 has
// no FP64 kind).  Each CTA regenerates its Y tile in shared memory from
// recurrence checkpoints (Y_k, Y_{k+1}) stored every 32 degrees, so tiles can
// start at any k and the recurrence of one tile is only 32 dependent steps.
#include "sht_internal.h"

#include <algorithm>
#include <type_traits>

namespace {

// FP64 tensor-core product of a 16 x 4 A tile and a 4 x 8 B tile
// (mma.sync m16n8k4): A rows g and g + 8 (a0, a1), C rows g (c0, c1) and
// g + 8 (c2, c3) for lane = 4 g + t; the registers of two row-adjacent
// 8 x 8 fragments.  Measured on B200 against m8n8k4 pairs: analysis 5 % faster
// at 64 fields, 14 % at 8; m16n8k8 (two k steps per instruction) was slower.
__device__ __forceinline__ void dmma16(double (&c0)[2], double (&c1)[2], double a0, double a1, double b)
{
	asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
	             : "+d"(c0[0]), "+d"(c0[1]), "+d"(c1[0]), "+d"(c1[1]) : "d"(a0), "d"(a1), "d"(b));
}

// Read-only load that does not allocate in L1: the streamed operands (F rows,
// coefficient rows, checkpoints) are read once per CTA, and keeping them out
// of L1 leaves it to the small per-row tables that every chunk's staging reads
// (recurrence coefficients, weights, cos and 1/sin of the latitudes).
__device__ __forceinline__ double2 ldg_stream(const double2* q)
{
	double2 v;
	asm("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(q));
	return v;
}



// ---------------------------------------------------------------------------
// Checkpoints: thread (t, im) runs the recurrence of order m at north row t and
// stores (Y_{seg*s}, Y_{seg*s+1}) for every segment s (seg = 8, 16 or 32).
// Y_0 = sin^m(theta) (sint_pow_n_ext, sht_legendre.c:110-139) and
// Y_1 = (c_1 x^2 + c_0) Y_0 (kernel_SH_to_spat.gen.c:303-315).
// Extended exponent: above degree ~1800, sin^m(theta) falls below the double
// range at latitudes where Y_k later grows to O(1).  The seed is formed as a
// mantissa times 2^E by binary powering with frexp normalisation, and the
// recurrence runs on scaled values y * 2^E (it is linear and homogeneous, so
// scaling by a power of two is exact) until the values have grown enough for
// E to be folded back to 0.  Each checkpoint stores y * 2^E as a plain double:
// a checkpoint that underflows is below 2^-1022 and stays below ~1e-280 over
// the next 32 steps, far under any threshold.  The reference keeps the same
// kind of scaled seed (sint_pow_n_ext, sht_legendre.c:109-139) and rescales
// its recurrence when values become significant (sht_legendre.c:159-187,
// sht_func.c:200-233).
#define CK_FOLD 600          // fold E into the values when E >= -CK_FOLD
#define CK_BIG 0x1p500       // rescale scaled values above this magnitude
__global__ void ck_kernel(int nlat_2, int mres, int seg, const double* __restrict__ x2g, const double* __restrict__ sing,
                          const double* __restrict__ c, MTables mt, const int* __restrict__ nseg, double2* __restrict__ ck)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	const int im = blockIdx.y;
	if (t >= nlat_2) return;
	const int m = im * mres;
	const double x2 = x2g[t];
	// sin^m = y0 * 2^E, y0 in [0.5, 1)
	double y0 = 1.0;
	int E = 0;
	{
		int be, te;
		double b = frexp(sing[t], &be);
		for (int n = m; n; n >>= 1) {
			if (n & 1) { y0 = frexp(y0 * b, &te); E += be + te; }
			b = frexp(b * b, &te); be = 2 * be + te;
		}
	}
	if (E >= -CK_FOLD) { y0 = ldexp(y0, E); E = 0; }
	const double* cc = c + mt.coff[im];
	double y1 = fma(cc[1], x2, cc[0]) * y0;
	const int ns = nseg[im];
	double2* out = ck + (long)mt.ckoff[im] * nlat_2 + t;
	for (int s = 0; s < ns; s++) {
		out[(long)s * nlat_2] = E ? make_double2(ldexp(y0, E), ldexp(y1, E)) : make_double2(y0, y1);
		const int kb = s * seg + 1;
		for (int j = 0; j < seg; j++) {
			const int k = kb + j;
			const double a = fma(cc[2 * k + 1], x2, cc[2 * k]);
			const double y2 = fma(a, y1, y0);
			y0 = y1;
			y1 = y2;
			if (E && fabs(y1) > CK_BIG) {
				if (E >= -CK_FOLD) { y0 = ldexp(y0, E); y1 = ldexp(y1, E); E = 0; }
				else { y0 *= 0x1p-500; y1 *= 0x1p-500; E += 500; }
			}
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
//
// CTA = (order im, 32 Ishioka rows k, 16 field-components): the degree window
// [2k0-1, 2k0+66] of each input array is staged in shared memory with
// coalesced loads, then every qq row segment is written contiguously.
#define PT_K 32
#define PT_F 16
#define PT_W 69          // window length (68 needed), odd stride in 16-byte units

__global__ void __launch_bounds__(256, 6) prep_synth_kernel(PrepParams p)
{
	__shared__ double2 win[2][PT_F][PT_W];
	__shared__ double cfs[2][PT_W];          // sin d/dtheta coupling (lo, hi) of the window's degrees
	__shared__ double xk[3 * PT_K];          // basis change X of the CTA's k rows
	__shared__ int s_comp[PT_F], s_f[PT_F];
	const int im = p.im0 + blockIdx.z;
	if (im > p.mlim) return;
	const int m = im * p.mres;
	const int kmax = (p.llim + 1 - m) / 2 + 1;
	const int k0 = blockIdx.x * PT_K;
	if (k0 >= kmax) return;
	const int nfc = p.nf * p.ncomp;
	const int fc0 = blockIdx.y * PT_F;
	const bool m0 = (m == 0);
	const int lrel_max = p.llim - m;
	const long off = (long)im * (2 * p.lmax + 2 - (im + 1) * p.mres) / 2 + m;   // LM(m, m)
	const int d0 = 2 * k0 - 1;
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int voff = p.mt.voff[im];
	if (tid < PT_F) {
		const int fc = fc0 + tid;
		const int comp = fc / p.nf;
		s_comp[tid] = (fc < nfc) ? comp : -1;
		s_f[tid] = fc - comp * p.nf;
	} else if (tid >= 32 && tid < 32 + PT_W) {
		const int i = tid - 32, d = d0 + i;
		cfs[0][i] = (d > 0 && d <= lrel_max + 1) ? p.stdt_lo[voff + d] : 0.0;
		cfs[1][i] = (d >= 0 && d <= lrel_max + 1) ? p.stdt_hi[voff + d] : 0.0;
	} else if (tid >= 128 && tid < 128 + 3 * PT_K) {
		const int e = tid - 128;
		xk[e] = (k0 + e / 3 <= kmax) ? p.xs[p.mt.xoff[im] + 3 * k0 + e] : 0.0;
	}
	// window of degrees d0 .. d0 + 68 of each (array, field-component): warp w
	// stages pairs w, w + 8, w + 16, w + 24 (array = pair / 16), lanes along
	// the degrees, two pairs at a time with all their loads issued before the
	// first store
	constexpr int NI = (PT_W + 31) / 32;
	#pragma unroll
	for (int h = 0; h < 2; h++) {
		double2 v[2][NI];
		#pragma unroll
		for (int qi = 0; qi < 2; qi++) {
			const int q = warp + 8 * (2 * h + qi), a = q / PT_F, fl = q % PT_F;
			const int fc = fc0 + fl;
			const double2* base = nullptr;
			if (fc < nfc) {
				const int comp = fc / p.nf, f = fc - comp * p.nf;
				base = (p.comp_type[comp] == 0) ? (a == 0 ? p.Q : nullptr) : (a == 0 ? p.S : p.T);
				if (base) base += off + (long)f * p.spec_dist;
			}
			#pragma unroll
			for (int u = 0; u < NI; u++) {
				const int d = d0 + lane + 32 * u;
				v[qi][u] = (base && lane + 32 * u < PT_W && d >= 0 && d <= lrel_max) ? base[d] : make_double2(0.0, 0.0);
			}
		}
		#pragma unroll
		for (int qi = 0; qi < 2; qi++) {
			const int q = warp + 8 * (2 * h + qi), a = q / PT_F, fl = q % PT_F;
			#pragma unroll
			for (int u = 0; u < NI; u++) {
				const int i = lane + 32 * u;
				if (i < PT_W) {
					double2 x = v[qi][u];
					if (m0) x.y = 0.0;
					win[a][fl][i] = x;
				}
			}
		}
	}
	__syncthreads();
	const double em = (p.msign < 0) ? -(double) m : (double) m;   // signed m (negative orders of the _ml transforms)
	for (int e = tid; e < PT_K * PT_F; e += blockDim.x) {
		const int kl = e / PT_F, fl = e - kl * PT_F;
		const int k = k0 + kl, fc = fc0 + fl;
		if (k >= kmax || fc >= nfc) continue;
		const int type = p.comp_type[s_comp[fl]];
		// fields from neg_from on carry the order -m (complex-field transforms)
		const int fld = s_f[fl];
		const double emf = (p.neg_from > 0 && fld >= p.neg_from) ? -em : em;
		const int i0 = 2 * kl + 1;                 // window index of degree 2k
		double2 q3[3];
		if (type == 0) {
			#pragma unroll
			for (int r = 0; r < 3; r++) q3[r] = win[0][fl][i0 + r];
		} else {
			// V = stdt S + i m T (type 1), W = -stdt T + i m S (type 2): the
			// coupled array at degrees d -/+ 1, the other one at d
			const int ac = (type == 1) ? 0 : 1;
			#pragma unroll
			for (int r = 0; r < 3; r++) {
				const int d = 2 * k + r;               // relative degree
				if (d > lrel_max + 1) { q3[r] = make_double2(0.0, 0.0); continue; }
				const double lo = cfs[0][i0 + r], hi = cfs[1][i0 + r];
				const double2 cm = win[ac][fl][i0 - 1 + r], cp = win[ac][fl][i0 + 1 + r], o0 = win[1 - ac][fl][i0 + r];
				if (type == 1)
					q3[r] = make_double2(lo * cm.x + hi * cp.x - emf * o0.y, lo * cm.y + hi * cp.y + emf * o0.x);
				else
					q3[r] = make_double2(-(lo * cm.x + hi * cp.x) - emf * o0.y, -(lo * cm.y + hi * cp.y) + emf * o0.x);
			}
		}
		const double x0 = xk[3 * kl], x1 = xk[3 * kl + 1], x2 = xk[3 * kl + 2];
		double* row = p.qq + (long)(p.mt.koff[im] + k) * p.ncol;
		const int ce = 16 * (fc >> 2) + 2 * (fc & 3);
		*reinterpret_cast<double2*>(row + ce) = make_double2(fma(x0, q3[0].x, x1 * q3[2].x), fma(x0, q3[0].y, x1 * q3[2].y));
		*reinterpret_cast<double2*>(row + ce + 8) = make_double2(x2 * q3[1].x, x2 * q3[1].y);
	}
}

// ---------------------------------------------------------------------------
// Analysis epilogue: Ishioka basis -> spectral coefficients
//   Q_{m+2k} = X0_k e_k + X1_{k-1} e_{k-1},  Q_{m+2k+1} = X2_k o_k
// (ishioka_to_SH, sht_private.h:345-374), and for vectors
//   S_l = -((MX V)_l + i m W_l) / (l(l+1)),  T_l = -(i m V_l - (MX W)_l) / (l(l+1))
// with MX = 2 cos + sin d/dtheta (SH_2scal_to_vect, sht_private.h:296-337).
// Degrees above llim and orders above mlim are written as zero (SHT_VAR_LTR).
//
// CTA = (order im, 64 degrees, 16 fields, output group): the k rows covering
// the degree tile plus one row of halo on each side are staged in shared
// memory for the (one or two) field-components of the group.
#define PE_J 64
#define PE_F 16
#define PE_R 36          // staged k rows: j0/2-2 .. j0/2+33
#define PE_S (2 * PE_F + 2)   // row stride in double2: 32 mod 128 bytes, so the 4 rows read by 8 lanes use distinct banks

// E[row][2 fl + 0] = even pair (re, im), [2 fl + 1] = odd pair, row = k - kb;
// Xs[3 row + c] = basis-change coefficients of k
__device__ __forceinline__ double2 ish_inv_s(const double2 (*E)[PE_S], const double* Xs, int kb, int fl, int j)
{
	if (j < 0) return make_double2(0.0, 0.0);
	const int r = (j >> 1) - kb;
	if ((j & 1) == 0) {
		const double2 e = E[r][2 * fl];
		const double x = Xs[3 * r];
		double2 q = make_double2(x * e.x, x * e.y);
		if (j > 1) {
			const double2 e1 = E[r - 1][2 * fl];
			const double x1 = Xs[3 * (r - 1) + 1];
			q.x = fma(x1, e1.x, q.x);
			q.y = fma(x1, e1.y, q.y);
		}
		return q;
	}
	const double2 o = E[r][2 * fl + 1];
	const double x2 = Xs[3 * r + 2];
	return make_double2(x2 * o.x, x2 * o.y);
}

__global__ void __launch_bounds__(256) post_analys_kernel(PrepParams p)
{
	constexpr int NE = PE_R * PE_F * 2, NU = (NE + 255) / 256;
	__shared__ double2 sv[PE_R][PE_S];     // first component of the group (Q, or V)
	__shared__ double2 sw[PE_R][PE_S];     // second component (W) for the vector group
	__shared__ double xs[3 * PE_R];
	const int im = p.im0 + blockIdx.z;
	const int m = im * p.mres;
	const int nl = p.lmax - m + 1;
	const int j0 = blockIdx.x * PE_J;
	if (j0 >= nl) return;
	const bool has_q = (p.comp_type[0] == 0);
	const int nft = (p.nf + PE_F - 1) / PE_F;
	const int g = blockIdx.y / nft;                       // 0: first group, 1: second group
	const int f0 = (blockIdx.y - g * nft) * PE_F;
	const bool scalar_group = has_q && g == 0;
	const bool zero_m = (im > p.mlim);
	const long off = (long)im * (2 * p.lmax + 2 - (im + 1) * p.mres) / 2 + m;
	const int kb = j0 / 2 - 2;
	const int nk = (p.llim + ((p.comp_type[0] | p.comp_type[1] | p.comp_type[2]) ? 1 : 0) - m) / 2 + 1;
	if (!zero_m) {
		const int cv = scalar_group ? 0 : (has_q ? 1 : 0);
		const long r0 = p.mt.koff[im];
		// all row loads of a thread are issued before the first is stored
		double2 v[NU], w[NU];
		#pragma unroll
		for (int u = 0; u < NU; u++) {
			const int e = threadIdx.x + 256 * u;
			const int r = e / (PE_F * 2), rem = e - r * PE_F * 2;
			const int fl = rem >> 1, eo = rem & 1;
			const int k = kb + r, f = f0 + fl;
			v[u] = make_double2(0.0, 0.0);
			w[u] = make_double2(0.0, 0.0);
			if (e < NE && k >= 0 && k < nk && f < p.nf) {
				const double* row = p.qq + (r0 + k) * p.ncol;
				const int fcv = cv * p.nf + f;
				v[u] = *reinterpret_cast<const double2*>(row + 16 * (fcv >> 2) + 2 * (fcv & 3) + 8 * eo);
				if (!scalar_group) {
					const int fcw = (cv + 1) * p.nf + f;
					w[u] = *reinterpret_cast<const double2*>(row + 16 * (fcw >> 2) + 2 * (fcw & 3) + 8 * eo);
				}
			}
		}
		// basis-change coefficients of the staged rows (3 (kmax + 1) entries per order)
		const int kx = (p.lmax + 1 - m) / 2 + 1;
		const double* X = p.xa + p.mt.xoff[im];
		for (int e = threadIdx.x; e < 3 * PE_R; e += blockDim.x) {
			const int k = kb + e / 3;
			xs[e] = (k >= 0 && k <= kx) ? X[3 * kb + e] : 0.0;
		}
		#pragma unroll
		for (int u = 0; u < NU; u++) {
			const int e = threadIdx.x + 256 * u;
			if (e < NE) {
				const int r = e / (PE_F * 2), c = e - r * PE_F * 2;
				sv[r][c] = v[u];
				sw[r][c] = w[u];
			}
		}
	}
	// vector coupling (lo, hi) of degrees j0 - 1 .. j0 + PE_J and 1 / (l (l + 1))
	// of the tile's degrees, shared by its fields
	__shared__ double vlo[PE_J + 2], vhi[PE_J + 2], vl2[PE_J];
	const int voff = p.mt.voff[im];
	if (!scalar_group) {
		for (int e = threadIdx.x; e < PE_J + 2; e += blockDim.x) {
			const int j = j0 - 1 + e;
			vlo[e] = (j > 0 && j < nl) ? p.van_lo[voff + j] : 0.0;
			vhi[e] = (j >= 0 && j < nl) ? p.van_hi[voff + j] : 0.0;
			if (e < PE_J) vl2[e] = (j0 + e < nl) ? p.l2[m + j0 + e] : 0.0;
		}
	}
	__syncthreads();
	const double em = (p.msign < 0) ? -(double) m : (double) m;   // signed m (negative orders of the _ml transforms)
	const int lane = threadIdx.x & 31;
	// a warp covers 32 consecutive degrees of one field: each lane forms its
	// own degree in the spectral basis and takes the neighbours (j -/+ 1) of
	// the vector formulas from the adjacent lanes
	for (int e = threadIdx.x; e < PE_J * PE_F; e += blockDim.x) {
		const int fl = e / PE_J, jl = e - fl * PE_J;
		const int j = j0 + jl, f = f0 + fl;
		const int l = m + j;
		const bool live = j < nl && f < p.nf;
		const long o = off + (long)f * p.spec_dist + j;
		const bool zero = zero_m || (l > p.llim);
		if (scalar_group) {
			if (!live) continue;
			double2 q = make_double2(0.0, 0.0);
			if (!zero) {
				q = ish_inv_s(sv, xs, kb, fl, j);
				if (m == 0) q.y = 0.0;
			}
			p.Qo[o] = q;
			continue;
		}
		const bool fv = !zero_m && f < p.nf && j < nl + 1;   // rows staged: degrees up to nl
		const double2 v0 = fv ? ish_inv_s(sv, xs, kb, fl, j) : make_double2(0.0, 0.0);
		const double2 w0 = fv ? ish_inv_s(sw, xs, kb, fl, j) : make_double2(0.0, 0.0);
		double2 vm, vp, wm, wp;
		vm.x = __shfl_up_sync(0xffffffffu, v0.x, 1); vm.y = __shfl_up_sync(0xffffffffu, v0.y, 1);
		wm.x = __shfl_up_sync(0xffffffffu, w0.x, 1); wm.y = __shfl_up_sync(0xffffffffu, w0.y, 1);
		vp.x = __shfl_down_sync(0xffffffffu, v0.x, 1); vp.y = __shfl_down_sync(0xffffffffu, v0.y, 1);
		wp.x = __shfl_down_sync(0xffffffffu, w0.x, 1); wp.y = __shfl_down_sync(0xffffffffu, w0.y, 1);
		if (!live) continue;
		double2 s = make_double2(0.0, 0.0), t = make_double2(0.0, 0.0);
		if (!zero) {
			if (lane == 0) { vm = ish_inv_s(sv, xs, kb, fl, j - 1); wm = ish_inv_s(sw, xs, kb, fl, j - 1); }
			if (lane == 31) { vp = ish_inv_s(sv, xs, kb, fl, j + 1); wp = ish_inv_s(sw, xs, kb, fl, j + 1); }
			const double lo = vlo[jl + 1];
			const double hi = vhi[jl + 1];
			const double l2 = vl2[jl];
			const double mxv_r = lo * vm.x + hi * vp.x, mxv_i = lo * vm.y + hi * vp.y;
			const double mxw_r = lo * wm.x + hi * wp.x, mxw_i = lo * wm.y + hi * wp.y;
			const double emf = (p.neg_from > 0 && f >= p.neg_from) ? -em : em;   // order -m fields
			s = make_double2(-(mxv_r - emf * w0.y) * l2, -(mxv_i + emf * w0.x) * l2);
			t = make_double2(-(-emf * v0.y - mxw_r) * l2, -(emf * v0.x - mxw_i) * l2);
			if (m == 0) { s.y = 0.0; t.y = 0.0; }
		}
		p.So[o] = s;
		p.To[o] = t;
	}
}

// ---------------------------------------------------------------------------
// Synthesis contraction.  CTA = (order im, 64 north theta rows, 64 columns).
// 8 warps as 2 (theta) x 4 (columns); a warp owns 32 rows x 16 columns = one
// group of 4 field-components, so each lane ends with (E_re, E_im, O_re, O_im)
// of one (row, field-component) and folds north/south itself.
#define SA_LD 68   // shared row stride in doubles: 4 mod 16 keeps fragment loads conflict-free

// WM = warps along the rows (2: 64 rows x 64 columns per CTA; 4: 128 rows x
// 32 columns, for calls with at most 8 field-components).
// RB: Fourier rows in per-block buffers (p.rb) instead of the plain F
template <int SEG, int WM, bool RB = false>
__device__ __forceinline__ void leg_synth_tile(const LegParams& p, int im, int tb, int nb)
{
	constexpr int WN = 8 / WM, BM = 32 * WM, BN = 16 * WN;
	__shared__ __align__(16) double As[LG_BK][BM + 4];   // [k][theta]; strides 4 mod 16:
	__shared__ __align__(16) double Bs[LG_BK][BN + 4];   // [k][col]    conflict-free fragment loads
	const int m = im * p.mres;
	const int t0 = tb * BM, c0 = nb * BN;
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int wm = warp / WN, wn = warp % WN;
	const int nk = (p.llim + p.vec_extra - m) / 2 + 1;
	const int tmm = p.mt.tm[im];

	double acc[4][2][2];
	#pragma unroll
	for (int i = 0; i < 4; i++)
		#pragma unroll
		for (int j = 0; j < 2; j++) { acc[i][j][0] = 0.0; acc[i][j][1] = 0.0; }

	// 8 x 8 fragments of this warp that carry results: rows in [tmm, nlat/2),
	// columns below ncol (the others are discarded by the epilogue)
	const int wr = t0 + wm * 32, wc = c0 + wn * 16;
	const int ri0 = min(4, max(0, (tmm - wr) / 8));
	const int ri1 = min(4, max(0, (p.nlat_2 - wr + 7) / 8));
	const int cj1 = min(2, max(0, (p.ncol - wc + 7) / 8));
	if (t0 + BM > tmm) {
		const double* cm = p.c + p.mt.coff[im];
		const double2* ckm = p.ck + (long)p.mt.ckoff[im] * p.nlat_2;
		const double* qrow = p.qq + (long)p.mt.koff[im] * p.ncol;
		// software pipeline: the B tile and checkpoint of chunk k0+32 are
		// loaded into registers while the tensor cores work on chunk k0
		constexpr int NBV = LG_BK * (BN / 2) / LG_THREADS;   // double2 per thread
		double2 bn[NBV];
		// generators: thread (row gr, segment sg = gj + u GPR) produces Y_k for
		// SEG consecutive k of the chunk from the checkpoint at its segment start
		constexpr int NSEGC = LG_BK / SEG;                    // segments per chunk
		constexpr int GPR = LG_THREADS / BM;                  // generator threads per row
		constexpr int SPT = (NSEGC + GPR - 1) / GPR;          // segments per generator thread
		double2 ckn[SPT];
		const int gr = tid % BM, gj = tid / BM;
		const int tg = t0 + gr;
		const bool gen = tg < p.nlat_2;
		const double x2 = gen ? p.x2[tg] : 0.0;
		auto load_b = [&](int k0) {
			#pragma unroll
			for (int u = 0; u < NBV; u++) {
				const int e = tid + u * LG_THREADS;
				const int kk = e / (BN / 2), cc2 = (e - kk * (BN / 2)) * 2;
				const int k = k0 + kk, col = c0 + cc2;
				bn[u] = (k < nk && col < p.ncol) ? ldg_stream(reinterpret_cast<const double2*>(qrow + (long)k * p.ncol + col))
				                                 : make_double2(0.0, 0.0);
			}
			#pragma unroll
			for (int u = 0; u < SPT; u++) {
				const int sg = gj + u * GPR;
				const int ks = k0 + sg * SEG;
				ckn[u] = (sg < NSEGC && gen && ks < nk) ? ldg_stream(ckm + (long)(ks / SEG) * p.nlat_2 + tg)
				                                       : make_double2(0.0, 0.0);
			}
		};
		load_b(0);
		for (int k0 = 0; k0 < nk; k0 += LG_BK) {
			#pragma unroll
			for (int u = 0; u < SPT; u++) {
				const int sg = gj + u * GPR;
				if (sg < NSEGC) {
					double y0 = ckn[u].x, y1 = ckn[u].y;
					As[sg * SEG][gr] = y0;
					As[sg * SEG + 1][gr] = y1;
					const double* cc = cm + 2 * (k0 + sg * SEG);
					#pragma unroll
					for (int j = 2; j < SEG; j++) {
						const double a = fma(cc[2 * j - 1], x2, cc[2 * j - 2]);
						const double y2 = fma(a, y1, y0);
						As[sg * SEG + j][gr] = y2;
						y0 = y1; y1 = y2;
					}
				}
			}
			#pragma unroll
			for (int u = 0; u < NBV; u++) {
				const int e = tid + u * LG_THREADS;
				const int kk = e / (BN / 2), cc2 = (e - kk * (BN / 2)) * 2;
				*reinterpret_cast<double2*>(&Bs[kk][cc2]) = bn[u];
			}
			__syncthreads();
			if (k0 + LG_BK < nk) load_b(k0 + LG_BK);
			const int kv = nk - k0;                      // steps of this chunk below nk
			// P0, P1: row-fragment pairs (0, 1) and (2, 3) computed; NJ column
			// fragments.  The choice is made once per warp with a branch: an MMA
			// switched off by a predicate still occupies the tensor pipe.
			auto mma_chunk = [&](auto P0, auto P1, auto NJ) {
				#pragma unroll
				for (int kk = 0; kk < LG_BK; kk += 4) {
					if (kk >= kv) break;                  // rows of Bs beyond nk are zero
					double a[4], b[2];
					#pragma unroll
					for (int i = 0; i < 4; i++)
						if ((i < 2 && P0.value) || (i >= 2 && P1.value)) a[i] = As[kk + (lane & 3)][wm * 32 + i * 8 + (lane >> 2)];
					#pragma unroll
					for (int j = 0; j < NJ.value; j++) b[j] = Bs[kk + (lane & 3)][wn * 16 + j * 8 + (lane >> 2)];
					#pragma unroll
					for (int j = 0; j < NJ.value; j++) {
						if constexpr (P0.value) dmma16(acc[0][j], acc[1][j], a[0], a[1], b[j]);
						if constexpr (P1.value) dmma16(acc[2][j], acc[3][j], a[2], a[3], b[j]);
					}
				}
			};
			// fragment pairs (i, i + 1) carry results when either row fragment does
			const bool p0 = ri0 <= 1 && ri1 > 0, p1 = ri0 <= 3 && ri1 > 2;
			using T = std::true_type;
			using F = std::false_type;
			using J1 = std::integral_constant<int, 1>;
			using J2 = std::integral_constant<int, 2>;
			if (cj1 == 2) {
				if (p0 && p1) mma_chunk(T{}, T{}, J2{});
				else if (p0) mma_chunk(T{}, F{}, J2{});
				else if (p1) mma_chunk(F{}, T{}, J2{});
			} else if (cj1 == 1) {
				if (p0 && p1) mma_chunk(T{}, T{}, J1{});
				else if (p0) mma_chunk(T{}, F{}, J1{});
				else if (p1) mma_chunk(F{}, T{}, J1{});
			}
			__syncthreads();
		}
	}
	// epilogue: fold hemispheres, apply 1/sin for vector components, store F
	const int fc = ((c0 + wn * 16) >> 4) * 4 + (lane & 3);
	if (fc >= p.nfc) return;
	const bool vec = (p.ctype[fc / p.nf] != 0) && !p.robert;
	double2* Ff = p.F + (long)fc * p.fstride + (long)im * p.nlat;     // plain layout (p.rb.n == 0)
	#pragma unroll
	for (int i = 0; i < 4; i++) {
		const int t = t0 + wm * 32 + i * 8 + (lane >> 2);
		if (t >= p.nlat_2) continue;
		const double cx = p.x[t];
		double nr = fma(cx, acc[i][1][0], acc[i][0][0]), ni = fma(cx, acc[i][1][1], acc[i][0][1]);
		double sr = fma(-cx, acc[i][1][0], acc[i][0][0]), si = fma(-cx, acc[i][1][1], acc[i][0][1]);
		if (t < tmm) { nr = ni = sr = si = 0.0; }
		if (vec) { const double s = p.sinv[t]; nr *= s; ni *= s; sr *= s; si *= s; }
		if (p.adjoint) {
			// adjoint of the analysis: row weight W_t(m) / (nphi (2 - delta_m0))
			const double s = p.w[t] * (m > 0 ? p.mpos_inv : 1.0) / (p.nphi * (m > 0 ? 2.0 : 1.0));
			nr *= s; ni *= s; sr *= s; si *= s;
		}
		const int rn = p.south_first ? p.nlat - 1 - t : t;
		const int rs = p.nlat - 1 - rn;
		if constexpr (!RB) {
			Ff[rn] = make_double2(nr, ni);
			Ff[rs] = make_double2(sr, si);
		} else {
			*fourier_row(p, fc, im, rn) = make_double2(nr, ni);
			*fourier_row(p, fc, im, rs) = make_double2(sr, si);
		}
	}
}

// ---------------------------------------------------------------------------
// Analysis contraction.  CTA = (order im, 64 k rows, 64 columns); the K loop
// runs over north theta rows in chunks of 32, starting at the polar threshold.
// The B operand is built while staging: G_even = w (F_N + F_S),
// G_odd = w cos(theta) (F_N - F_S) (kernel_spat_to_SH.gen.c:485-491), times
// 1/sin(theta) for vector components (1/sin^2 in Robert form).
#define AA_LD 36   // As row stride (k rows x 32 theta): 4 mod 16

// WM = warps along the k rows (2: 64 k x 64 columns per CTA; 4: 128 k x 32
// columns, for calls with at most 8 field-components).
template <int SEG, int WM, bool RB = false>
__device__ __forceinline__ void leg_analys_tile(const LegParams& p, int im, int kb, int nb)
{
	constexpr int WN = 8 / WM, BM = 32 * WM, BN = 16 * WN;
	__shared__ __align__(16) double As[BM][AA_LD];       // [k][theta]
	__shared__ __align__(16) double Bs[LG_BK][BN + 4];   // [theta][col]
	const int m = im * p.mres;
	const int k0 = kb * BM, c0 = nb * BN;
	const int nk = (p.llim + p.vec_extra - m) / 2 + 1;
	if (k0 >= nk) return;
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int wm = warp / WN, wn = warp % WN;
	const int tmm = p.mt.tm[im];
	const double wfac = (m > 0) ? p.mpos_inv : 1.0;
	const double* cm = p.c + p.mt.coff[im];
	const double2* ckm = p.ck + (long)p.mt.ckoff[im] * p.nlat_2;
	const int fc0 = c0 / 4;
	// 8 x 8 fragments of this warp that carry results: k below nk, columns
	// below ncol (the others are not stored)
	const int ki1 = min(4, max(0, (nk - k0 - wm * 32 + 7) / 8));
	const int cj1 = min(2, max(0, (p.ncol - c0 - wn * 16 + 7) / 8));

	double acc[4][2][2];
	#pragma unroll
	for (int i = 0; i < 4; i++)
		#pragma unroll
		for (int j = 0; j < 2; j++) { acc[i][j][0] = 0.0; acc[i][j][1] = 0.0; }

	// software pipeline: F values and checkpoints of the next theta chunk are
	// loaded into registers while the tensor cores work on the current one
	constexpr int NBF = LG_BK * (BN / 4) / LG_THREADS;   // (theta, field-component) items per thread
	double2 fnn[NBF], fsn[NBF];
	// generators: thread (theta gtt, segment sg = gsg + u GPT) produces Y_k
	// for SEG consecutive k of the CTA's k rows from the checkpoint at its
	// segment start
	constexpr int NSG = BM / SEG;                         // segments per tile
	constexpr int GPT = LG_THREADS / LG_BK;               // generator threads per theta
	constexpr int SPT = (NSG + GPT - 1) / GPT;            // segments per generator thread
	double2 ckn[SPT];
	const int gtt = tid % LG_BK, gsg = tid / LG_BK;
	// vector flag of each staging item's field-component (fixed per thread)
	bool vecn[NBF];
	#pragma unroll
	for (int u = 0; u < NBF; u++) {
		const int fc = fc0 + (tid + u * LG_THREADS) / LG_BK;
		vecn[u] = fc < p.nfc && p.ctype[fc / p.nf] != 0;
	}
	auto load_next = [&](int tt0) {
		#pragma unroll
		for (int u = 0; u < NBF; u++) {
			const int e = tid + u * LG_THREADS;
			const int tt = e % LG_BK, fl = e / LG_BK;
			const int t = tt0 + tt, fc = fc0 + fl;
			fnn[u] = make_double2(0.0, 0.0); fsn[u] = make_double2(0.0, 0.0);
			if (t < p.nlat_2 && t >= tmm && fc < p.nfc) {
				const int rn = p.south_first ? p.nlat - 1 - t : t;
				const int rs = p.nlat - 1 - rn;
				if constexpr (!RB) {
					const double2* Ff = p.F + (long)fc * p.fstride + (long)im * p.nlat;
					fnn[u] = ldg_stream(Ff + rn);
					fsn[u] = ldg_stream(Ff + rs);
				} else {
					fnn[u] = ldg_stream(fourier_row(p, fc, im, rn));
					fsn[u] = ldg_stream(fourier_row(p, fc, im, rs));
				}
			}
		}
		const int t = tt0 + gtt;
		#pragma unroll
		for (int u = 0; u < SPT; u++) {
			const int sg = gsg + u * GPT, gks = k0 + sg * SEG;
			ckn[u] = (sg < NSG && t < p.nlat_2 && gks < nk) ? ldg_stream(ckm + (long)(gks / SEG) * p.nlat_2 + t)
			                                               : make_double2(0.0, 0.0);
		}
	};
	// recurrence coefficients of the CTA's k rows, staged once (rows at or
	// beyond nk get zeros: their results are not stored)
	__shared__ double cs[2 * BM];
	for (int e = tid; e < 2 * BM; e += LG_THREADS) cs[e] = (k0 + e / 2 < nk) ? cm[2 * k0 + e] : 0.0;
	__syncthreads();
	const int tstart = (tmm / LG_BK) * LG_BK;
	if (tstart < p.nlat_2) load_next(tstart);
	for (int tt0 = tstart; tt0 < p.nlat_2; tt0 += LG_BK) {
		{
			const int t = tt0 + gtt;
			const double x2 = (t < p.nlat_2) ? p.x2[t] : 0.0;
			#pragma unroll
			for (int u = 0; u < SPT; u++) {
				const int sg = gsg + u * GPT, gks = k0 + sg * SEG;
				if (sg >= NSG) break;
				double y0 = ckn[u].x, y1 = ckn[u].y;
				double* a = &As[sg * SEG][gtt];
				a[0] = y0;
				a[AA_LD] = y1;
				if (gks < nk) {
					const double* cc = cs + 2 * sg * SEG;
					#pragma unroll
					for (int j = 2; j < SEG; j++) {
						const double aa = fma(cc[2 * j - 1], x2, cc[2 * j - 2]);
						const double y2 = fma(aa, y1, y0);
						a[j * AA_LD] = y2;
						y0 = y1; y1 = y2;
					}
				} else {
					for (int j = 2; j < SEG; j++) a[j * AA_LD] = 0.0;
				}
			}
		}
		#pragma unroll
		for (int u = 0; u < NBF; u++) {
			const int e = tid + u * LG_THREADS;
			const int tt = e % LG_BK, fl = e / LG_BK;
			const int t = tt0 + tt, fc = fc0 + fl;
			double er = 0.0, ei = 0.0, orr = 0.0, oi = 0.0;
			if (t < p.nlat_2 && fc < p.nfc) {
				// adjoint of the synthesis: no quadrature weight, factor nphi (2 - delta_m0)
				double w = p.adjoint ? p.nphi * (m > 0 ? 2.0 : 1.0) : p.w[t] * wfac;
				if (vecn[u]) {
					double s = p.sinv[t];
					if (p.robert) s *= s;
					w *= s;
				}
				const double wo = w * p.x[t];
				const double2 fn = fnn[u], fs = fsn[u];
				er = w * (fn.x + fs.x);  ei = w * (fn.y + fs.y);
				orr = wo * (fn.x - fs.x); oi = wo * (fn.y - fs.y);
			}
			// columns swizzled by row: bits 1-2 of the column XOR (row / 4) % 4, so
			// that the 16 rows a half-warp stores hit distinct banks; the fragment
			// loads read 4 consecutive rows (one swizzle) and stay conflict-free
			const int cb = (16 * (fl >> 2) + 2 * (fl & 3)) ^ (2 * ((tt >> 2) & 3));
			*reinterpret_cast<double2*>(&Bs[tt][cb]) = make_double2(er, ei);
			*reinterpret_cast<double2*>(&Bs[tt][cb + 8]) = make_double2(orr, oi);
		}
		__syncthreads();
		if (tt0 + LG_BK < p.nlat_2) load_next(tt0 + LG_BK);
		// NP row-fragment pairs and NJ column fragments, chosen once per warp
		// with a branch (a predicated-off MMA still occupies the tensor pipe)
		auto mma_chunk = [&](auto NP, auto NJ) {
			#pragma unroll
			for (int kk = 0; kk < LG_BK; kk += 4) {
				double a[4], b[2];
				#pragma unroll
				for (int i = 0; i < 2 * NP.value; i++) a[i] = As[wm * 32 + i * 8 + (lane >> 2)][kk + (lane & 3)];
				#pragma unroll
				for (int j = 0; j < NJ.value; j++)
					b[j] = Bs[kk + (lane & 3)][(wn * 16 + j * 8 + (lane >> 2)) ^ (2 * ((kk >> 2) & 3))];
				#pragma unroll
				for (int j = 0; j < NJ.value; j++)
					#pragma unroll
					for (int i = 0; i < 2 * NP.value; i += 2) dmma16(acc[i][j], acc[i + 1][j], a[i], a[i + 1], b[j]);
			}
		};
		using N1 = std::integral_constant<int, 1>;
		using N2 = std::integral_constant<int, 2>;
		if (ki1 > 2) {
			if (cj1 == 2) mma_chunk(N2{}, N2{});
			else if (cj1 == 1) mma_chunk(N2{}, N1{});
		} else if (ki1 > 0) {
			if (cj1 == 2) mma_chunk(N1{}, N2{});
			else if (cj1 == 1) mma_chunk(N1{}, N1{});
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

// Single-plan kernels: blockIdx.y = order - p.im0, blockIdx.x = (row tile, column tile).
template <int SEG, int WM, bool RB>
__global__ void __launch_bounds__(LG_THREADS, WM == 1 ? 2 : 3) leg_synth_kernel(LegParams p)
{
	const int ntb = (p.nlat_2 + 32 * WM - 1) / (32 * WM);
	leg_synth_tile<SEG, WM, RB>(p, p.im0 + blockIdx.y, blockIdx.x % ntb, blockIdx.x / ntb);
}

template <int SEG, int WM, bool RB>
__global__ void __launch_bounds__(LG_THREADS, WM == 1 ? 2 : 3) leg_analys_kernel(LegParams p, int nkb)
{
	leg_analys_tile<SEG, WM, RB>(p, p.im0 + blockIdx.y, blockIdx.x % nkb, blockIdx.x / nkb);
}

// Persistent multi-plan kernels: CTAs (one wave) take work items (plan,
// order, row or k tile, column tile) from a queue in decreasing cost order,
// so plans of different lmax share one launch and balance over the SMs.
template <int SEG, bool SYNTH>
__global__ void __launch_bounds__(LG_THREADS, 3)
leg_multi_kernel(const LegParams* __restrict__ plist, const int4* __restrict__ work, int nwork, int* __restrict__ counter)
{
	__shared__ int wi;
	for (;;) {
		if (threadIdx.x == 0) wi = atomicAdd(counter, 1);
		__syncthreads();
		const int w = wi;
		__syncthreads();
		if (w >= nwork) break;
		const int4 it = work[w];
		if (SYNTH) leg_synth_tile<SEG, 2>(plist[it.x], it.y, it.z, it.w);
		else leg_analys_tile<SEG, 2>(plist[it.x], it.y, it.z, it.w);
	}
}

} // namespace

// ---------------------------------------------------------------------------
void launch_checkpoints(shtns_cfg s, cudaStream_t st)
{
	std::vector<int> nseg(s->mmax + 1);
	for (int im = 0; im <= s->mmax; im++) nseg[im] = (s->kmax_h[im] + s->ckseg - 1) / s->ckseg;
	int* d_nseg = nullptr;
	if (!shtb_cuda_ok(cudaMalloc(&d_nseg, sizeof(int) * nseg.size()), "checkpoint table")) return;
	cudaMemcpyAsync(d_nseg, nseg.data(), sizeof(int) * nseg.size(), cudaMemcpyHostToDevice, st);
	dim3 grid((s->nlat_2 + 127) / 128, s->mmax + 1);
	ck_kernel<<<grid, 128, 0, st>>>(s->nlat_2, s->mres, s->ckseg, s->d_x2, s->d_s, s->d_c, s->mt, d_nseg, s->d_ck);
	shtb_count_launch();
	shtb_cuda_ok(cudaGetLastError(), "checkpoint kernel");
	cudaStreamSynchronize(st);
	cudaFree(d_nseg);
}

void launch_prep_synth(const PrepParams& p, cudaStream_t st)
{
	const int nfc = p.nf * p.ncomp;
	const int kmax0 = (p.llim + 1) / 2 + 1;
	dim3 grid((kmax0 + PT_K - 1) / PT_K, (nfc + PT_F - 1) / PT_F, p.mlim + 1 - p.im0);
	prep_synth_kernel<<<grid, 256, 0, st>>>(p);
	shtb_count_launch();
}

namespace {

template <int WM>
void launch_leg_synth_wm(const LegParams& p, cudaStream_t st)
{
	constexpr int BM = 32 * WM, BN = 16 * (8 / WM);
	const int ntb = (p.nlat_2 + BM - 1) / BM;
	const int nnb = (p.ncol + BN - 1) / BN;
	dim3 grid(ntb * nnb, p.mlim + 1 - p.im0);
	switch (p.ckseg) {
		case 8: if (p.rb.n) leg_synth_kernel<8, WM, true><<<grid, LG_THREADS, 0, st>>>(p);
		        else leg_synth_kernel<8, WM, false><<<grid, LG_THREADS, 0, st>>>(p); break;
		case 16: if (p.rb.n) leg_synth_kernel<16, WM, true><<<grid, LG_THREADS, 0, st>>>(p);
		         else leg_synth_kernel<16, WM, false><<<grid, LG_THREADS, 0, st>>>(p); break;
		default: if (p.rb.n) leg_synth_kernel<32, WM, true><<<grid, LG_THREADS, 0, st>>>(p);
		         else leg_synth_kernel<32, WM, false><<<grid, LG_THREADS, 0, st>>>(p); break;
	}
}

template <int WM>
void launch_leg_analys_wm(const LegParams& p, int kmax_all, cudaStream_t st)
{
	constexpr int BM = 32 * WM, BN = 16 * (8 / WM);
	const int nkb = (kmax_all + BM - 1) / BM;
	const int nnb = (p.ncol + BN - 1) / BN;
	dim3 grid(nkb * nnb, p.mlim + 1 - p.im0);
	switch (p.ckseg) {
		case 8: if (p.rb.n) leg_analys_kernel<8, WM, true><<<grid, LG_THREADS, 0, st>>>(p, nkb);
		        else leg_analys_kernel<8, WM, false><<<grid, LG_THREADS, 0, st>>>(p, nkb); break;
		case 16: if (p.rb.n) leg_analys_kernel<16, WM, true><<<grid, LG_THREADS, 0, st>>>(p, nkb);
		         else leg_analys_kernel<16, WM, false><<<grid, LG_THREADS, 0, st>>>(p, nkb); break;
		default: if (p.rb.n) leg_analys_kernel<32, WM, true><<<grid, LG_THREADS, 0, st>>>(p, nkb);
		         else leg_analys_kernel<32, WM, false><<<grid, LG_THREADS, 0, st>>>(p, nkb); break;
	}
}

} // namespace

// Tile shape (p.tile_wm, warps along the rows): 1 = 32 x 128, 2 = 64 x 64,
// 4 = 128 x 32.  Automatic (0): calls with at most 32 GEMM columns (8
// field-components) use 128 x 32, which leaves no column padding; wider
// calls 64 x 64.
static int tile_wm(const LegParams& p)
{
	if (p.tile_wm == 1 || p.tile_wm == 2 || p.tile_wm == 4) return p.tile_wm;
	return p.ncol <= 32 ? 4 : 2;
}

void launch_leg_synth(const LegParams& p, cudaStream_t st)
{
	if (leg_simt_selected(p, true)) { launch_leg_synth_simt(p, st); shtb_count_launch(); return; }
	switch (tile_wm(p)) {
		case 1: launch_leg_synth_wm<1>(p, st); break;
		case 4: launch_leg_synth_wm<4>(p, st); break;
		default: launch_leg_synth_wm<2>(p, st); break;
	}
	shtb_count_launch();
}

void launch_leg_analys(const LegParams& p, int kmax_all, cudaStream_t st)
{
	if (leg_simt_selected(p, false)) { launch_leg_analys_simt(p, kmax_all, st); shtb_count_launch(); return; }
	switch (tile_wm(p)) {
		case 1: launch_leg_analys_wm<1>(p, kmax_all, st); break;
		case 4: launch_leg_analys_wm<4>(p, kmax_all, st); break;
		default: launch_leg_analys_wm<2>(p, kmax_all, st); break;
	}
	shtb_count_launch();
}

void launch_post_analys_m(const PrepParams& p, int mmax, cudaStream_t st)
{
	const int ngroups = (p.comp_type[0] == 0) ? 1 + (p.ncomp > 1 ? 1 : 0) : 1;
	const int nft = (p.nf + PE_F - 1) / PE_F;
	dim3 grid((p.lmax + 1 + PE_J - 1) / PE_J, nft * ngroups, mmax + 1 - p.im0);
	post_analys_kernel<<<grid, 256, 0, st>>>(p);
	shtb_count_launch();
}

void launch_leg_multi(const LegParams* d_plist, const int4* d_work, int nwork, int* d_counter, int ckseg, bool synth,
                      int nctas, cudaStream_t st)
{
	const int grid = std::max(1, std::min(nwork, nctas));
	cudaMemsetAsync(d_counter, 0, sizeof(int), st);
	switch (ckseg) {
		case 8:
			if (synth) leg_multi_kernel<8, true><<<grid, LG_THREADS, 0, st>>>(d_plist, d_work, nwork, d_counter);
			else leg_multi_kernel<8, false><<<grid, LG_THREADS, 0, st>>>(d_plist, d_work, nwork, d_counter);
			break;
		case 16:
			if (synth) leg_multi_kernel<16, true><<<grid, LG_THREADS, 0, st>>>(d_plist, d_work, nwork, d_counter);
			else leg_multi_kernel<16, false><<<grid, LG_THREADS, 0, st>>>(d_plist, d_work, nwork, d_counter);
			break;
		default:
			if (synth) leg_multi_kernel<32, true><<<grid, LG_THREADS, 0, st>>>(d_plist, d_work, nwork, d_counter);
			else leg_multi_kernel<32, false><<<grid, LG_THREADS, 0, st>>>(d_plist, d_work, nwork, d_counter);
			break;
	}
	shtb_count_launch();
}
