// SIMT FP64 Legendre kernels for calls with few field-components (1 to 4).
//
// The tensor-core tiles (sht_legendre.cu) multiply the on-the-fly Y tile by 16
// GEMM columns per group of 4 field-components; with one field 12 of the 16
// columns are padding.  On sm_100a the FP64 FMA pipe has the throughput of the
// FP64 tensor path, so for one to four field-components these kernels do the
// minimum work instead: per (row, k) two FMAs of recurrence and four FMAs per
// field-component, with Y never leaving registers in the synthesis.
//
// Same recurrence, checkpoints and coefficient layout as the tensor-core
// kernels (the reference's SHT/kernel_SH_to_spat.gen.c:388-441 and
// kernel_spat_to_SH.gen.c:485-598): Y_k for k = seg*SEG and seg*SEG+1 comes
// from the checkpoint table, Y_{k} = (c_{2k-1} x^2 + c_{2k-2}) Y_{k-1} + Y_{k-2}
// inside a segment; qq[k][16*(fc/4) + 2*(fc%4) + 8*odd + {re, im}].
#include "sht_internal.h"

#include <algorithm>

namespace {

// ---------------------------------------------------------------------------
// Synthesis.  CTA = (2*nt north rows, order); thread = rows ta and ta + nt.
// Per chunk of 64 k the recurrence constants and the coefficients of the
// chunk are staged in shared memory; every thread reads the same k at the same
// time (broadcast loads).
#define SS_KC 64                       // k per staged chunk (a multiple of every SEG)

// address of a Fourier row: plain layout, or per-block buffers when RB
template <bool RB>
__device__ __forceinline__ double2* simt_row(const LegParams& p, int fc, int im, int row)
{
	if constexpr (RB) return fourier_row(p, fc, im, row);
	else return p.F + (long)fc * p.fstride + (long)im * p.nlat + row;
}

template <int NFC>
__device__ __forceinline__ void simt_acc(double (&a)[NFC][4], const double* cs, double y)
{
	#pragma unroll
	for (int f = 0; f < NFC; f++) {
		const double2 e = *reinterpret_cast<const double2*>(cs + 2 + 4 * f);
		const double2 o = *reinterpret_cast<const double2*>(cs + 4 + 4 * f);
		a[f][0] = fma(y, e.x, a[f][0]);
		a[f][1] = fma(y, e.y, a[f][1]);
		a[f][2] = fma(y, o.x, a[f][2]);
		a[f][3] = fma(y, o.y, a[f][3]);
	}
}

// fold hemispheres, scale, store the two Fourier rows of north row t
template <int NFC, bool RB>
__device__ __forceinline__ void simt_synth_store(const LegParams& p, int im, int tmm, int t, const double (&a)[NFC][4])
{
	if (t >= p.nlat_2) return;
	const int m = im * p.mres;
	const double cx = p.x[t];
	const int rn = p.south_first ? p.nlat - 1 - t : t;
	const int rs = p.nlat - 1 - rn;
	#pragma unroll
	for (int f = 0; f < NFC; f++) {
		double nr = fma(cx, a[f][2], a[f][0]), ni = fma(cx, a[f][3], a[f][1]);
		double sr = fma(-cx, a[f][2], a[f][0]), si = fma(-cx, a[f][3], a[f][1]);
		if (t < tmm) { nr = ni = sr = si = 0.0; }
		if (p.ctype[f / p.nf] != 0 && !p.robert) {
			const double s = p.sinv[t];
			nr *= s; ni *= s; sr *= s; si *= s;
		}
		if (p.adjoint) {
			const double s = p.w[t] * (m > 0 ? p.mpos_inv : 1.0) / (p.nphi * (m > 0 ? 2.0 : 1.0));
			nr *= s; ni *= s; sr *= s; si *= s;
		}
		*simt_row<RB>(p, f, im, rn) = make_double2(nr, ni);
		*simt_row<RB>(p, f, im, rs) = make_double2(sr, si);
	}
}

template <int SEG, int NFC, bool RB>
__global__ void __launch_bounds__(128) leg_synth_simt_kernel(LegParams p)
{
	constexpr int W = 2 + 4 * NFC;     // staged doubles per k: (c_{2k-2}, c_{2k-1}), then per fc E re, E im, O re, O im
	__shared__ __align__(16) double cs[SS_KC * W];
	const int im = p.im0 + blockIdx.y;
	const int m = im * p.mres;
	const int nt = blockDim.x;
	const int tmm = p.mt.tm[im];
	const int nk = (p.llim + p.vec_extra - m) / 2 + 1;
	const int tb = blockIdx.x * 2 * nt;
	const int ta = tb + threadIdx.x, tc = ta + nt;
	const bool la = ta < p.nlat_2 && ta >= tmm, lc = tc < p.nlat_2 && tc >= tmm;
	double aa[NFC][4], ac[NFC][4];
	#pragma unroll
	for (int f = 0; f < NFC; f++)
		#pragma unroll
		for (int u = 0; u < 4; u++) { aa[f][u] = 0.0; ac[f][u] = 0.0; }
	if (min(tb + 2 * nt, p.nlat_2) > tmm) {          // uniform: some row of the CTA is above the polar threshold
		const double* cm = p.c + p.mt.coff[im];
		const double2* ckm = p.ck + (long)p.mt.ckoff[im] * p.nlat_2;
		const double* qrow = p.qq + (long)p.mt.koff[im] * p.ncol;
		const double xa = la ? p.x2[ta] : 0.0, xc = lc ? p.x2[tc] : 0.0;
		const double2 z = make_double2(0.0, 0.0);
		double2 na = la ? __ldg(ckm + ta) : z, nc = lc ? __ldg(ckm + tc) : z;
		for (int k0 = 0; k0 < nk; k0 += SS_KC) {
			__syncthreads();
			for (int e = threadIdx.x; e < SS_KC * W; e += nt) {
				const int kk = e / W, w = e - kk * W, k = k0 + kk;
				double v = 0.0;
				if (k < nk) {
					if (w < 2) {
						v = (k >= 2) ? __ldg(cm + 2 * k - 2 + w) : 0.0;
					} else {
						const int f = (w - 2) >> 2, u = (w - 2) & 3;
						v = __ldg(qrow + (long)k * p.ncol + 16 * (f >> 2) + 2 * (f & 3) + ((u & 2) ? 8 : 0) + (u & 1));
					}
				}
				cs[e] = v;
			}
			__syncthreads();
			const int kend = min(SS_KC, nk - k0);
			for (int s0 = 0; s0 < kend; s0 += SEG) {
				const int sg = (k0 + s0) / SEG;
				double ya0 = na.x, ya1 = na.y, yc0 = nc.x, yc1 = nc.y;
				const bool more = k0 + s0 + SEG < nk;     // checkpoint of the next segment, loaded ahead
				na = (la && more) ? __ldg(ckm + (long)(sg + 1) * p.nlat_2 + ta) : z;
				nc = (lc && more) ? __ldg(ckm + (long)(sg + 1) * p.nlat_2 + tc) : z;
				const double* c = cs + s0 * W;
				simt_acc<NFC>(aa, c, ya0);
				simt_acc<NFC>(ac, c, yc0);
				if (s0 + 1 < kend) {
					simt_acc<NFC>(aa, c + W, ya1);
					simt_acc<NFC>(ac, c + W, yc1);
				}
				#pragma unroll
				for (int j = 2; j < SEG; j++) {
					if (s0 + j >= kend) break;
					const double* cj = c + j * W;
					const double2 r = *reinterpret_cast<const double2*>(cj);
					const double fa = fma(r.y, xa, r.x), fc = fma(r.y, xc, r.x);
					const double ya2 = fma(fa, ya1, ya0), yc2 = fma(fc, yc1, yc0);
					ya0 = ya1; ya1 = ya2;
					yc0 = yc1; yc1 = yc2;
					simt_acc<NFC>(aa, cj, ya2);
					simt_acc<NFC>(ac, cj, yc2);
				}
			}
		}
	}
	simt_synth_store<NFC, RB>(p, im, tmm, ta, aa);
	simt_synth_store<NFC, RB>(p, im, tmm, tc, ac);
}

// ---------------------------------------------------------------------------
// Analysis.  CTA = (order, block of 2*nt k); thread = k rows kb0 + tid and
// kb0 + tid + nt.  Per chunk of 16 north rows: the threads generate Y for the
// chunk's rows and the block's k into shared memory (thread = row tid % 16,
// segments tid / 16 + u * nt / 16) and stage G = w (F_N + F_S),
// w cos (F_N - F_S) of the chunk; then every thread sums its two k over the 16
// rows.  No reduction across threads.
#define SA_TB 16                       // north rows per chunk
#define SA_NT 128                      // largest block

template <int SEG, int NFC, bool RB>
__global__ void __launch_bounds__(SA_NT) leg_analys_simt_kernel(LegParams p)
{
	constexpr int SPT = 32 / SEG;      // segments per generator thread: (2 nt / SEG) / (nt / 16)
	constexpr int GW = 4 * NFC;
	__shared__ __align__(16) double As[SA_TB * (2 * SA_NT + 1)];   // [row][k], odd row stride
	__shared__ __align__(16) double Gs[SA_TB * GW];
	const int im = p.im0 + blockIdx.y;
	const int m = im * p.mres;
	const int nt = blockDim.x, kbs = 2 * nt, ld = kbs + 1;
	const int nk = (p.llim + p.vec_extra - m) / 2 + 1;
	const int kb0 = blockIdx.x * kbs;
	if (kb0 >= nk) return;
	const int tid = threadIdx.x;
	const int tmm = p.mt.tm[im];
	const double wfac = (m > 0) ? p.mpos_inv : 1.0;
	const double* cm = p.c + p.mt.coff[im];
	const double2* ckm = p.ck + (long)p.mt.ckoff[im] * p.nlat_2;
	const int gr = tid & (SA_TB - 1), gs = tid / SA_TB, ngs = nt / SA_TB;
	double acc[2][NFC][4];
	#pragma unroll
	for (int u = 0; u < 2; u++)
		#pragma unroll
		for (int f = 0; f < NFC; f++)
			#pragma unroll
			for (int v = 0; v < 4; v++) acc[u][f][v] = 0.0;

	const int tstart = (tmm / SA_TB) * SA_TB;
	double2 ckn[SPT];
	// G items (row e % 16, field-component e / 16) for e = tid + i nt < 16 NFC:
	// at most 2 per thread (nt >= 32, NFC <= 4); their Fourier values, loaded ahead
	double2 fn[2], fs[2];
	auto load_next = [&](int tt0) {
		const int t = tt0 + gr;
		#pragma unroll
		for (int u = 0; u < SPT; u++) {
			const int ks = kb0 + (gs + u * ngs) * SEG;
			ckn[u] = (t < p.nlat_2 && t >= tmm && ks < nk) ? __ldg(ckm + (long)(ks / SEG) * p.nlat_2 + t)
			                                              : make_double2(0.0, 0.0);
		}
		#pragma unroll
		for (int i = 0; i < 2; i++) {
			const int e = tid + i * nt, gt = e % SA_TB, gf = e / SA_TB;
			const int tg = tt0 + gt;
			fn[i] = make_double2(0.0, 0.0); fs[i] = fn[i];
			if (gf < NFC && tg < p.nlat_2 && tg >= tmm) {
				const int rn = p.south_first ? p.nlat - 1 - tg : tg;
				const int rs = p.nlat - 1 - rn;
				fn[i] = __ldg(simt_row<RB>(p, gf, im, rn));
				fs[i] = __ldg(simt_row<RB>(p, gf, im, rs));
			}
		}
	};
	if (tstart < p.nlat_2) load_next(tstart);
	bool vg[2];                                     // vector flag of each staging item's field-component
	#pragma unroll
	for (int i = 0; i < 2; i++) {
		const int gf = (tid + i * nt) / SA_TB;
		vg[i] = gf < NFC && p.ctype[gf / p.nf] != 0;
	}
	for (int tt0 = tstart; tt0 < p.nlat_2; tt0 += SA_TB) {
		// phase 1: Y of (row gr, this thread's segments) and G of (row gt, component gf)
		{
			const int t = tt0 + gr;
			const double x2 = (t < p.nlat_2) ? p.x2[t] : 0.0;
			#pragma unroll
			for (int u = 0; u < SPT; u++) {
				const int sl = gs + u * ngs;             // segment within the block
				const int ks = kb0 + sl * SEG;
				double* a = As + gr * ld + sl * SEG;
				double y0 = ckn[u].x, y1 = ckn[u].y;
				a[0] = y0;
				a[1] = y1;
				if (ks < nk) {
					const double* cc = cm + 2 * ks;
					#pragma unroll
					for (int j = 2; j < SEG; j++) {
						const double aa = fma(__ldg(cc + 2 * j - 1), x2, __ldg(cc + 2 * j - 2));
						const double y2 = fma(aa, y1, y0);
						a[j] = y2;
						y0 = y1; y1 = y2;
					}
				} else {
					#pragma unroll
					for (int j = 2; j < SEG; j++) a[j] = 0.0;
				}
			}
			#pragma unroll
			for (int i = 0; i < 2; i++) {
				const int e = tid + i * nt, gt = e % SA_TB, gf = e / SA_TB;
				if (gf >= NFC) continue;
				const int tg = tt0 + gt;
				double er = 0.0, ei = 0.0, orr = 0.0, oi = 0.0;
				if (tg < p.nlat_2) {
					double w = p.adjoint ? p.nphi * (m > 0 ? 2.0 : 1.0) : p.w[tg] * wfac;
					if (vg[i]) {
						double s = p.sinv[tg];
						if (p.robert) s *= s;
						w *= s;
					}
					const double wo = w * p.x[tg];
					er = w * (fn[i].x + fs[i].x);  ei = w * (fn[i].y + fs[i].y);
					orr = wo * (fn[i].x - fs[i].x); oi = wo * (fn[i].y - fs[i].y);
				}
				double* g = Gs + gt * GW + 4 * gf;
				*reinterpret_cast<double2*>(g) = make_double2(er, ei);
				*reinterpret_cast<double2*>(g + 2) = make_double2(orr, oi);
			}
		}
		__syncthreads();
		if (tt0 + SA_TB < p.nlat_2) load_next(tt0 + SA_TB);
		// phase 2: the thread's two k over the chunk's rows
		#pragma unroll 4
		for (int r = 0; r < SA_TB; r++) {
			const double y0 = As[r * ld + tid], y1 = As[r * ld + tid + nt];
			#pragma unroll
			for (int f = 0; f < NFC; f++) {
				const double2 ge = *reinterpret_cast<const double2*>(Gs + r * GW + 4 * f);
				const double2 go = *reinterpret_cast<const double2*>(Gs + r * GW + 4 * f + 2);
				acc[0][f][0] = fma(y0, ge.x, acc[0][f][0]); acc[0][f][1] = fma(y0, ge.y, acc[0][f][1]);
				acc[0][f][2] = fma(y0, go.x, acc[0][f][2]); acc[0][f][3] = fma(y0, go.y, acc[0][f][3]);
				acc[1][f][0] = fma(y1, ge.x, acc[1][f][0]); acc[1][f][1] = fma(y1, ge.y, acc[1][f][1]);
				acc[1][f][2] = fma(y1, go.x, acc[1][f][2]); acc[1][f][3] = fma(y1, go.y, acc[1][f][3]);
			}
		}
		__syncthreads();
	}
	double* qrow = p.qq + (long)p.mt.koff[im] * p.ncol;
	#pragma unroll
	for (int u = 0; u < 2; u++) {
		const int k = kb0 + tid + u * nt;
		if (k >= nk) continue;
		#pragma unroll
		for (int f = 0; f < NFC; f++) {
			double* q = qrow + (long)k * p.ncol + 16 * (f >> 2) + 2 * (f & 3);
			*reinterpret_cast<double2*>(q) = make_double2(acc[u][f][0], acc[u][f][1]);
			*reinterpret_cast<double2*>(q + 8) = make_double2(acc[u][f][2], acc[u][f][3]);
		}
	}
}

// ---------------------------------------------------------------------------
// Analysis of one field-component with the partial sums in registers.
// CTA = (order, block of 16 k), 64 threads; every thread takes north rows
// tmm + tid, tmm + tid + 64, ... and for each runs the recurrence over the
// block (from the checkpoint of its segment, advancing to the block start
// when the block starts inside a segment) and accumulates Y_k G for its rows:
// 4 x 16 = 64 sums per thread.  They are reduced once per CTA: a butterfly
// reduce-scatter inside each warp (lane L ends with sums 2L and 2L+1), then
// across the two warps in shared memory.  Measured on B200 against the
// shared-memory kernel above: faster for one component when the checkpoints
// are 16 or 32 apart or the grid has at most 1024 rows (2x at lmax 127, 1.5x at
// 511, 1.15x at 4095), slower at lmax 1023 (checkpoints 8 apart) and for two
// components.
#define SR_NT 64
#define SR_NV 64                       // partial sums per thread

template <int SEG, bool RB>
__global__ void __launch_bounds__(SR_NT) leg_analys_reg_kernel(LegParams p)
{
	constexpr int NFC = 1;
	constexpr int KB = 16;                             // k per block
	constexpr int NSB = (KB > SEG) ? KB / SEG : 1;     // checkpoints per row and block
	constexpr int NC = SEG + KB + 2;                   // recurrence constants staged per block
	__shared__ double2 cs[NC];
	__shared__ double red[SR_NT / 32][SR_NV];
	constexpr int nt = SR_NT;
	const int im = p.im0 + blockIdx.y;
	const int m = im * p.mres;
	const int nk = (p.llim + p.vec_extra - m) / 2 + 1;
	const int kb0 = blockIdx.x * KB;
	if (kb0 >= nk) return;
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int tmm = p.mt.tm[im];
	const int s0 = (kb0 / SEG) * SEG;                  // first segment start of the block
	const double* cm = p.c + p.mt.coff[im];
	for (int i = tid; i < NC; i += nt) {
		const int k = s0 + i;
		cs[i] = (k >= 2 && k < nk) ? make_double2(__ldg(cm + 2 * k - 2), __ldg(cm + 2 * k - 1)) : make_double2(0.0, 0.0);
	}
	__syncthreads();
	const double2* ckm = p.ck + (long)p.mt.ckoff[im] * p.nlat_2;
	const double wfac = (m > 0) ? p.mpos_inv : 1.0;
	double v[SR_NV];
	#pragma unroll
	for (int i = 0; i < SR_NV; i++) v[i] = 0.0;

	// the loads of row t + 128 are issued before the work of row t
	double2 nfn[NFC], nfs[NFC], nck[NSB];
	double nw = 0.0, nx = 0.0, nx2 = 0.0, nsv = 0.0;
	auto load_row = [&](int t) {
		if (t >= p.nlat_2) return;
		const int rn = p.south_first ? p.nlat - 1 - t : t;
		const int rs = p.nlat - 1 - rn;
		#pragma unroll
		for (int f = 0; f < NFC; f++) {
			nfn[f] = __ldg(simt_row<RB>(p, f, im, rn));
			nfs[f] = __ldg(simt_row<RB>(p, f, im, rs));
		}
		#pragma unroll
		for (int b = 0; b < NSB; b++) {
			const int ks = (NSB > 1) ? kb0 + b * SEG : s0;
			nck[b] = (ks < nk) ? __ldg(ckm + (long)(ks / SEG) * p.nlat_2 + t) : make_double2(0.0, 0.0);
		}
		nw = p.adjoint ? 0.0 : __ldg(p.w + t);
		nx = __ldg(p.x + t);
		nx2 = __ldg(p.x2 + t);
		nsv = __ldg(p.sinv + t);
	};
	bool vf[NFC];                                   // vector flag per field-component
	#pragma unroll
	for (int f = 0; f < NFC; f++) vf[f] = p.ctype[f / p.nf] != 0;
	load_row(tmm + tid);
	for (int t = tmm + tid; t < p.nlat_2; t += nt) {
		// G of this row: w (F_N + F_S), w cos (F_N - F_S) per field-component
		double g[NFC][4];
		const double x2 = nx2;
		double2 ckr[NSB];
		#pragma unroll
		for (int f = 0; f < NFC; f++) {
			double w = p.adjoint ? p.nphi * (m > 0 ? 2.0 : 1.0) : nw * wfac;
			if (vf[f]) {
				double sv = nsv;
				if (p.robert) sv *= sv;
				w *= sv;
			}
			const double wo = w * nx;
			const double2 fn = nfn[f], fs = nfs[f];
			g[f][0] = w * (fn.x + fs.x);  g[f][1] = w * (fn.y + fs.y);
			g[f][2] = wo * (fn.x - fs.x); g[f][3] = wo * (fn.y - fs.y);
		}
		#pragma unroll
		for (int b = 0; b < NSB; b++) ckr[b] = nck[b];
		load_row(t + nt);
		#pragma unroll
		for (int b = 0; b < NSB; b++) {
			const int ks = (NSB > 1) ? kb0 + b * SEG : s0;           // segment start
			if (ks >= nk) break;
			const double2 ck = ckr[b];
			double ya = ck.x, yb = ck.y;                               // Y_ks, Y_ks+1
			int ci = ks - s0 + 2;                                      // constants of Y_{ks+2}
			if (NSB == 1) {
				// advance from the segment start to the block start
				for (int k = ks; k < kb0; k++, ci++) {
					const double2 c = cs[ci];
					const double y2 = fma(fma(c.y, x2, c.x), yb, ya);
					ya = yb; yb = y2;
				}
			}
			constexpr int JN = (NSB > 1) ? SEG : KB;
			#pragma unroll
			for (int jj = 0; jj < JN; jj++) {
				const int j = b * JN + jj;                             // k = kb0 + j
				#pragma unroll
				for (int f = 0; f < NFC; f++) {
					#pragma unroll
					for (int u = 0; u < 4; u++) v[(j * NFC + f) * 4 + u] = fma(ya, g[f][u], v[(j * NFC + f) * 4 + u]);
				}
				if (jj + 1 < JN) {
					const double2 c = cs[ci + jj];
					const double y2 = fma(fma(c.y, x2, c.x), yb, ya);
					ya = yb; yb = y2;
				}
			}
		}
	}
	// reduce-scatter over the warp: after the level of stride s, lanes with
	// bit s set hold the upper half of the remaining sums
	#pragma unroll
	for (int s = 16, n = SR_NV / 2; s >= 1; s >>= 1, n >>= 1) {
		const bool up = (lane & s) != 0;
		#pragma unroll
		for (int i = 0; i < n; i++) {
			const double send = up ? v[i] : v[i + n];
			const double keep = up ? v[i + n] : v[i];
			v[i] = keep + __shfl_xor_sync(0xffffffffu, send, s);
		}
	}
	red[warp][2 * lane] = v[0];
	red[warp][2 * lane + 1] = v[1];
	__syncthreads();
	for (int e = tid; e < SR_NV; e += nt) {
		double sum = 0.0;
		#pragma unroll
		for (int w = 0; w < nt / 32; w++) sum += red[w][e];
		const int j = e / (4 * NFC), f = (e / 4) % NFC, u = e & 3;
		const int k = kb0 + j;
		if (k < nk)
			p.qq[((long)p.mt.koff[im] + k) * p.ncol + 16 * (f >> 2) + 2 * (f & 3) + ((u & 2) ? 8 : 0) + (u & 1)] = sum;
	}
}

template <int SEG, bool RB>
void synth_seg_rb(const LegParams& p, dim3 grid, int nt, cudaStream_t st)
{
	switch (p.nfc) {
		case 1: leg_synth_simt_kernel<SEG, 1, RB><<<grid, nt, 0, st>>>(p); break;
		case 2: leg_synth_simt_kernel<SEG, 2, RB><<<grid, nt, 0, st>>>(p); break;
		case 3: leg_synth_simt_kernel<SEG, 3, RB><<<grid, nt, 0, st>>>(p); break;
		default: leg_synth_simt_kernel<SEG, 4, RB><<<grid, nt, 0, st>>>(p); break;
	}
}

template <int SEG>
void synth_seg(const LegParams& p, dim3 grid, int nt, cudaStream_t st)
{
	if (p.rb.n) synth_seg_rb<SEG, true>(p, grid, nt, st);
	else synth_seg_rb<SEG, false>(p, grid, nt, st);
}

template <int SEG, bool RB>
void analys_seg_rb(const LegParams& p, dim3 grid, int nt, cudaStream_t st)
{
	switch (p.nfc) {
		case 1: leg_analys_simt_kernel<SEG, 1, RB><<<grid, nt, 0, st>>>(p); break;
		case 2: leg_analys_simt_kernel<SEG, 2, RB><<<grid, nt, 0, st>>>(p); break;
		case 3: leg_analys_simt_kernel<SEG, 3, RB><<<grid, nt, 0, st>>>(p); break;
		default: leg_analys_simt_kernel<SEG, 4, RB><<<grid, nt, 0, st>>>(p); break;
	}
}

template <int SEG>
void analys_seg(const LegParams& p, dim3 grid, int nt, cudaStream_t st)
{
	if (p.rb.n) analys_seg_rb<SEG, true>(p, grid, nt, st);
	else analys_seg_rb<SEG, false>(p, grid, nt, st);
}

} // namespace

// Calls with 1..4 field-components take the SIMT kernels when the tile option
// asks for them (8) or, automatically (0), up to 4 components in the synthesis
// and 3 in the analysis (measured on B200 at lmax 511, 1023 and 4095: with 4
// components the tensor-core analysis tiles are faster below lmax 4095).
bool leg_simt_selected(const LegParams& p, bool synth)
{
	if (p.nfc < 1 || p.nfc > 4) return false;
	if (p.tile_wm == 8) return true;
	return p.tile_wm == 0 && p.nfc <= (synth ? 4 : 3);
}

void launch_leg_synth_simt(const LegParams& p, cudaStream_t st)
{
	const int half = (p.nlat_2 + 1) / 2;
	const int nt = std::min(128, std::max(32, (half + 31) / 32 * 32));
	dim3 grid((p.nlat_2 + 2 * nt - 1) / (2 * nt), p.mlim + 1 - p.im0);
	switch (p.ckseg) {
		case 8: synth_seg<8>(p, grid, nt, st); break;
		case 16: synth_seg<16>(p, grid, nt, st); break;
		default: synth_seg<32>(p, grid, nt, st); break;
	}
}

template <int SEG>
void analys_reg_seg(const LegParams& p, int kmax_all, cudaStream_t st)
{
	dim3 grid((kmax_all + 15) / 16, p.mlim + 1 - p.im0);
	if (p.rb.n) leg_analys_reg_kernel<SEG, true><<<grid, SR_NT, 0, st>>>(p);
	else leg_analys_reg_kernel<SEG, false><<<grid, SR_NT, 0, st>>>(p);
}

void launch_leg_analys_simt(const LegParams& p, int kmax_all, cudaStream_t st)
{
	if (p.nfc == 1 && (p.ckseg >= 16 || p.nlat_2 <= 512)) {
		switch (p.ckseg) {
			case 8: analys_reg_seg<8>(p, kmax_all, st); break;
			case 16: analys_reg_seg<16>(p, kmax_all, st); break;
			default: analys_reg_seg<32>(p, kmax_all, st); break;
		}
		return;
	}
	// block of 2 nt k: the smallest of 32, 64, 128 threads that covers kmax_all
	int nt = 32;
	while (nt < SA_NT && 2 * nt < kmax_all) nt *= 2;
	dim3 grid((kmax_all + 2 * nt - 1) / (2 * nt), p.mlim + 1 - p.im0);
	switch (p.ckseg) {
		case 8: analys_seg<8>(p, grid, nt, st); break;
		case 16: analys_seg<16>(p, grid, nt, st); break;
		default: analys_seg<32>(p, grid, nt, st); break;
	}
}
