// Split-precision Legendre stages from a precomputed table of Legendre
// values, on the INT8 tensor cores (tcgen05.mma kind::i8).
//
// The per-order contractions of the FP64 transform,
//   synthesis  out[t, c] = sum_k Y_k(t) q[k, c]      (t: north latitude)
//   analysis   q[k, c]   = sum_t Y_k(t) G[t, c]      (G: weighted N/S fold of F)
// are evaluated as exact integer sums of products of 8-bit digits
// (Ozaki-style splitting, with integer instead of floating-point slices):
//   Y_k(t)  = 2^(e_t + 2) sum_i a_i[t,k] 2^(-8(i+1))      e_t: exponent of max_k |Y_k(t)|
//   q[k, c] = 2^(f_c + 2) sum_j b_j[k,c] 2^(-8(j+1))      f_c: exponent of max_k |q[k, c]|
// a_i, b_j in [-128, 127] (the leading digit in [-65, 65]: values are scaled
// below 1/4).  Products with i + j < NS are kept; D_s = sum_{i+j=s} sum_k
// a_i b_j accumulates exactly in INT32 tensor memory (|a_i b_j| <= 2^14, at
// most NS * 3072 terms per accumulator below 2^31), and
//   out = 2^(e_t + f_c + 4) sum_s 2^(-8(s+2)) D_s
// is formed in FP64 once per tile.  NS = 7 keeps 54 bits.  For the analysis
// the row scale moves to the other operand: G'[t, c] = 2^(e_t + 2) G[t, c] is
// split with its own column exponent, so the same integer digits of Y serve
// both directions.
//
// The digits of Y (the table, built once per plan on first use from the
// recurrence checkpoints with the FP64 kernels' own arithmetic) are stored in
// 16 KB digit-blocks of 128 latitudes x 128 Ishioka steps, as 8 x 16-byte core
// matrices: core matrix (a, b) = latitudes 8a..8a+7, steps 16b..16b+15 at byte
// (16 b + a) 128, step fastest.  The synthesis reads a block as the K-major A
// operand (M = latitudes, K = steps), the analysis reads the same bytes as
// the MN-major A operand (M = steps, K = latitudes).  Per order the table
// keeps the latitude tiles at or beyond the polar threshold and the step
// blocks up to the plan's last step (degree lmax + 1).  Below the turning
// point of each latitude (degrees l < m / sin(theta)) the Legendre values
// decay exponentially; the build records, per order and latitude tile, the
// first step block holding a nonzero digit, and the contraction skips the
// blocks before it (their digits are all zero, so nothing is lost).
//
// Kernel shape (both directions, one CTA per 128-row tile of one order and 32
// GEMM columns = 8 field-components; 192 threads, two CTAs per SM):
//   warp 0, one thread: bulk copies (cp.async.bulk, no multicast) of the
//     coefficient (or weighted Fourier) digit stack of the next 128-step (or
//     128-latitude) block and of its NS digit-blocks of Y into a ring of
//     shared-memory slots, completion on mbarriers;
//   warp 1, one thread: per digit-block i, tcgen05.mma (M = 128, N = 32 (NS -
//     i), K = 32) into accumulator columns 32 i .. 32 NS - 1 against the stacked
//     digits j < NS - i; tcgen05.commit frees the slot;
//   warps 2-5: read the NS INT32 accumulators (tcgen05.ld), combine them in
//     FP64 and store F (synthesis: folded hemispheres, as leg_synth_tile) or
//     the Ishioka-basis coefficients (analysis).
// The two 256-column accumulator buffers alternate between items, so the
// epilogue of one item overlaps the products of the next; the analysis (with
// two or more column tiles) instead gives each item two column tiles (one
// table read for both, their accumulators in the two halves of tensor
// memory).
// Every mbarrier wait is bounded (about one second by %globaltimer); a wait
// that gives up records an error flag (shtns_b200_kernel_errors), the CTA
// waits (bounded) for the copies and products it issued, frees its tensor
// memory and returns.
//
// The reference computes these sums in FP64 on the CPU
// (SHT/kernel_SH_to_spat.gen.c:388-409, kernel_spat_to_SH.gen.c:502-598);
// this path is a project extension.
#include "sht_internal.h"
#include "sht_ptx.h"

#include <algorithm>
#include <cstdint>

namespace {

constexpr int PB_T = 128;                  // latitudes per digit-block and per synthesis CTA
constexpr int PB_K = 128;                  // Ishioka steps per digit-block and per analysis CTA
constexpr int PB_BYTES = PB_T * PB_K;      // one digit-block: 16 KB
constexpr int PT_NC = 32;                  // GEMM columns per CTA
constexpr int PT_THREADS = 192;
// CT: 32-column tiles per work item.  CT = 1: two accumulator buffers in
// tensor memory (the epilogue of one item overlaps the products of the
// next); CT = 2: each digit-block of the table is read once for two column
// tiles, whose accumulators fill the one 512-column buffer (tile c at column
// 256 c), so the epilogue does not overlap the products (the analysis, see
// contract()).
template <int NS, int CT = 1>
struct PtLayout {
	static constexpr int RA = (CT == 1) ? 8 : 6;               // digit-block slots of the copy ring
	static constexpr int B_BYTES = NS * PT_NC * 128;          // digit stack of one block: NS x 32 rows x 128 bytes
	static constexpr int B_SLOT = CT * B_BYTES;               // stacks of the item's column tiles
	static constexpr int B_GRP = NS * (PT_NC / 8) * 128;      // bytes between 16-step (or 16-latitude) groups of a stack
	static constexpr int A_OFF = 0;
	static constexpr int B_OFF = RA * PB_BYTES;
	static constexpr int BAR_OFF = B_OFF + 2 * B_SLOT;
	static constexpr int NBAR = 2 * RA + 2 + 2 + 2 + 2 + 1;    // fullA, emptyA, fullB, emptyB, tfull, tempty, drain
	static constexpr int BE_OFF = BAR_OFF + 8 * NBAR + 16;     // column exponents of the current item, per epilogue warp
	static constexpr int TOTAL = BE_OFF + 4 * CT * PT_NC * 4;
	static constexpr int ACC_COLS = 256;                        // one accumulator buffer / tile (NS x 32 used)
	static_assert(PT_NC * NS <= ACC_COLS, "accumulators exceed a buffer");
	static_assert(CT == 1 || CT == 2, "column tiles per item");
	static_assert(TOTAL + 1024 <= 227 * 1024, "shared memory");
};

// ---- PTX helpers (mbarriers and bulk copies: sht_ptx.h) ----
using namespace shtb_ptx;

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// shared-memory matrix descriptor, no swizzle; lbo / sbo in bytes (K-major:
// lbo between core matrices along K, sbo between 8-row groups along M/N;
// MN-major: lbo between 8-row groups along K, sbo between 16-byte chunks
// along M/N)
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
	uint64_t d = 0;
	d |= (uint64_t)((addr >> 4) & 0x3FFF);
	d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
	d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
	d |= (uint64_t)1 << 46;            // descriptor version of sm_100
	return d;
}

// instruction descriptor of kind::i8: signed x signed -> INT32; a_mn / b_mn:
// 1 for an MN-major operand
__host__ __device__ constexpr uint32_t idesc_i8(int M, int N, int a_mn, int b_mn)
{
	return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t) a_mn << 15) | ((uint32_t) b_mn << 16) |
	       ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
	asm volatile("{\n\t.reg .pred p;\n\t"
	             "setp.ne.b32 p, %4, 0;\n\t"
	             "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
	             :: "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc) : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar)
{
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
	             :: "r"(smem_u32(bar)) : "memory");
}

// 16 consecutive INT32 columns of this warp's 32 lanes
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, int* v)
{
	uint32_t r[16];
	asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
	             "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
	             : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
	               "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
	             : "r"(taddr));
	asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
	#pragma unroll
	for (int i = 0; i < 16; i++) v[i] = (int) r[i];
}

// 2^n as a double from its exponent bits (normal range; ldexp otherwise)
__device__ __forceinline__ double pow2(int n)
{
	if (n >= -1022 && n <= 1023) return __longlong_as_double((long long)(n + 1023) << 52);
	return ldexp(1.0, n);
}

// NS balanced 8-bit digits of v, |v| < 1/4: v ~ sum_i d_i 2^(-8(i+1)), d_i in
// [-128, 127] for i >= 1 and d_0 in [-65, 65].  The value is rounded once to
// an integer multiple of 2^(-8 NS) (exact FP64 scaling, one conversion), then
// the digits are peeled from the bottom with sign-extended bytes.
template <int NS>
__device__ __forceinline__ void digits(double v, int* d)
{
	long long T = __double2ll_rn(v * (double)(1ull << (8 * NS)));
	#pragma unroll
	for (int i = NS - 1; i >= 1; i--) {
		const int lo = (int)(signed char)(T & 0xFF);
		d[i] = lo;
		T = (T - lo) >> 8;
	}
	d[0] = (int) T;
}

// sixteen values of one column (or row) as NS 16-byte digit rows
template <int NS>
__device__ __forceinline__ void pack16(const double (&v)[16], uint4 (&w)[NS])
{
	uint32_t acc[NS][4];
	#pragma unroll
	for (int i = 0; i < NS; i++) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0u;
	#pragma unroll
	for (int e = 0; e < 16; e++) {
		int d[NS];
		digits<NS>(v[e], d);
		#pragma unroll
		for (int i = 0; i < NS; i++) acc[i][e >> 2] |= ((uint32_t) d[i] & 0xFFu) << (8 * (e & 3));
	}
	#pragma unroll
	for (int i = 0; i < NS; i++) w[i] = make_uint4(acc[i][0], acc[i][1], acc[i][2], acc[i][3]);
}

struct PtabRef {
	const uint8_t* tab;
	const long* toff;        // per order: first digit-block
	const long* koff;        // per order: first 128-step block (coefficient stacks)
	const long* voff;        // per order: first kept latitude tile (Fourier stacks)
	const int* t0;           // per order: first latitude tile kept
	const int* kf;           // per (order, kept tile) at voff: first step block with a nonzero digit
	const short* yexp;       // row exponents [im][north row]
	int ntb;                 // latitude tiles of the grid
	int lmax;                // table steps of order m: (lmax + 1 - m) / 2 + 1
};

__device__ __forceinline__ int tab_kblocks(const PtabRef& t, int m) { return ((t.lmax + 1 - m) / 2 + 1 + PB_K - 1) / PB_K; }

// ---------------------------------------------------------------------------
// Table: CTA (latitude tile tb, order im), one thread per latitude.  Y_k is
// regenerated from the checkpoint at the start of every SEG-step segment with
// the FP64 kernels' operations (leg_synth_tile), on values scaled by
// 2^-(e_t + 2) (a power of two: the recurrence commutes with it).
template <int NS>
__global__ void __launch_bounds__(PB_T) ptab_build_kernel(PtabRef t, int nlat_2, int mres, int seg,
                                                          const double* __restrict__ x2g, const double* __restrict__ c,
                                                          MTables mt, const double2* __restrict__ ck, uint8_t* __restrict__ tab)
{
	const int tb = blockIdx.x, im = blockIdx.y;
	const int t0 = t.t0[im];
	if (tb < t0) return;
	const int m = im * mres;
	const int kmax = (t.lmax + 1 - m) / 2 + 1;
	const int nbk = (kmax + PB_K - 1) / PB_K;
	const int r = threadIdx.x;
	const int row = tb * PB_T + r;
	const bool live = row < nlat_2;
	const int e = live ? t.yexp[(long)im * nlat_2 + row] : -2000;
	const double rsc = (live && e > -1000) ? ldexp(1.0, -(e + 2)) : 0.0;
	const double x2 = live ? x2g[row] : 0.0;
	const double* cc = c + mt.coff[im];
	const double2* ckm = ck + (long)mt.ckoff[im] * nlat_2 + (live ? row : 0);
	uint8_t* base = tab + (t.toff[im] + (long)(tb - t0) * NS * nbk) * PB_BYTES + (r >> 3) * 128 + (r & 7) * 16;
	__shared__ int first_nz;
	if (r == 0) first_nz = nbk;
	__syncthreads();
	int my_first = nbk;
	double y0 = 0.0, y1 = 0.0;
	for (int kg = 0; kg < nbk * (PB_K / 16); kg++) {
		double v[16];
		#pragma unroll
		for (int e16 = 0; e16 < 16; e16++) {
			const int k = kg * 16 + e16;
			double y = 0.0;
			if (rsc != 0.0 && k < kmax) {
				const int j = k % seg;
				if (j == 0) {
					const double2 q = __ldg(ckm + (long)(k / seg) * nlat_2);
					y0 = q.x * rsc; y1 = q.y * rsc;
					y = y0;
				} else if (j == 1) {
					y = y1;
				} else {
					const double a = fma(__ldg(cc + 2 * k - 1), x2, __ldg(cc + 2 * k - 2));
					const double y2 = fma(a, y1, y0);
					y0 = y1; y1 = y2;
					y = y2;
				}
			}
			v[e16] = y;
		}
		uint4 w[NS];
		pack16<NS>(v, w);
		const int kb = kg / (PB_K / 16), b = kg % (PB_K / 16);
		#pragma unroll
		for (int i = 0; i < NS; i++) {
			*reinterpret_cast<uint4*>(base + ((long) i * nbk + kb) * PB_BYTES + b * 16 * 128) = w[i];
			if ((w[i].x | w[i].y | w[i].z | w[i].w) && kb < my_first) my_first = kb;
		}
	}
	atomicMin(&first_nz, my_first);
	__syncthreads();
	if (r == 0) const_cast<int*>(t.kf)[t.voff[im] + (tb - t0)] = first_nz;
}

// ---------------------------------------------------------------------------
// Coefficient digit stacks (synthesis B operand).  CTA (column tile ct, order
// im): column exponents f_c over the call's steps, then per 128-step block a
// stack of NS x 32 rows (row n = 32 j + column, digit j) x 128 steps, K-major:
// 16-step group g at g B_GRP, row n at (n / 8) 128 + (n % 8) 16.
template <int NS>
__global__ void __launch_bounds__(256) ptab_qslice_kernel(PtabRef t, const double* __restrict__ qq, int ncol, MTables mt,
                                                          int llim, int vec_extra, int mres, int nct,
                                                          uint8_t* __restrict__ bs, int* __restrict__ bexp)
{
	using L = PtLayout<NS>;
	__shared__ double red[8][PT_NC];
	__shared__ double colsc[PT_NC];
	const int ct = blockIdx.x, im = blockIdx.y;
	const int m = im * mres;
	const int nk = (llim + vec_extra - m) / 2 + 1;
	const int nbk = (nk + PB_K - 1) / PB_K;
	const double* qrow = qq + (long)mt.koff[im] * ncol;
	const int tid = threadIdx.x;
	{
		const int cl = tid & 31, kr = tid >> 5;
		const int col = ct * PT_NC + cl;
		double mx = 0.0;
		if (col < ncol)
			for (int k = kr; k < nk; k += 8) mx = fmax(mx, fabs(qrow[(long)k * ncol + col]));
		red[kr][cl] = mx;
	}
	__syncthreads();
	if (tid < PT_NC) {
		double mx = 0.0;
		for (int q = 0; q < 8; q++) mx = fmax(mx, red[q][tid]);
		int e = 0;
		if (mx > 0.0) frexp(mx, &e);
		colsc[tid] = (mx > 0.0) ? ldexp(1.0, -(e + 2)) : 0.0;
		bexp[(long)im * (nct * PT_NC) + ct * PT_NC + tid] = (mx > 0.0) ? e : -2000;
	}
	__syncthreads();
	for (int u = tid; u < nbk * (PB_K / 16) * PT_NC; u += 256) {
		const int cl = u & 31, kgl = u >> 5;
		const int col = ct * PT_NC + cl;
		double v[16];
		#pragma unroll
		for (int e16 = 0; e16 < 16; e16++) {
			const int k = kgl * 16 + e16;
			v[e16] = (k < nk && col < ncol) ? qrow[(long)k * ncol + col] * colsc[cl] : 0.0;
		}
		uint4 w[NS];
		pack16<NS>(v, w);
		const int kb = kgl / (PB_K / 16), g = kgl % (PB_K / 16);
		uint8_t* blk = bs + ((t.koff[im] + kb) * nct + ct) * (long) L::B_BYTES + (long) g * L::B_GRP;
		#pragma unroll
		for (int j = 0; j < NS; j++) {
			const int n = PT_NC * j + cl;
			*reinterpret_cast<uint4*>(blk + (n >> 3) * 128 + (n & 7) * 16) = w[j];
		}
	}
}

// Weighted Fourier digit stacks (analysis B operand).  CTA (column tile ct,
// order im): G'[t, c] = 2^(e_t + 2) G[t, c] with G_even = w (F_N + F_S), G_odd
// = w cos(theta) (F_N - F_S) as leg_analys_tile builds it (zero below the
// polar threshold), column exponents g_c over the kept latitudes, then per
// latitude tile a stack of NS x 32 rows x 128 latitudes, K-major (16-latitude
// groups at B_GRP).  Pass 1 (column maxima) and the value staging of pass 2
// run with consecutive threads on consecutive latitudes of one
// field-component (coalesced rows of F); pass 2 stages a tile's 32 x 128
// values in shared memory and packs the digits of (column, 16 latitudes)
// per thread.
__device__ __forceinline__ void gvalues(const PtabRef& t, const LegParams& p, int im, int fc, int row, double wfac, int m,
                                        double (&g)[4])
{
	g[0] = g[1] = g[2] = g[3] = 0.0;
	if (fc >= p.nfc || row < p.mt.tm[im] || row >= p.nlat_2) return;
	const int e = t.yexp[(long) im * p.nlat_2 + row];
	if (e <= -1000) return;
	double w = p.adjoint ? p.nphi * (m > 0 ? 2.0 : 1.0) : p.w[row] * wfac;
	if (p.ctype[fc / p.nf] != 0) {
		double s = p.sinv[row];
		if (p.robert) s *= s;
		w *= s;
	}
	w = ldexp(w, e + 2);
	const double wo = w * p.x[row];
	const int rn = p.south_first ? p.nlat - 1 - row : row;
	const int rs = p.nlat - 1 - rn;
	const double2* Ff = p.F + (long) fc * p.fstride + (long) im * p.nlat;
	const double2 fn = __ldg(Ff + rn), fs = __ldg(Ff + rs);
	g[0] = w * (fn.x + fs.x); g[1] = w * (fn.y + fs.y);
	g[2] = wo * (fn.x - fs.x); g[3] = wo * (fn.y - fs.y);
}

template <int NS>
__global__ void __launch_bounds__(256) ptab_gslice_kernel(PtabRef t, LegParams p, int nct, uint8_t* __restrict__ bs,
                                                          int* __restrict__ bexp)
{
	using L = PtLayout<NS>;
	__shared__ double vals[PT_NC][PB_T + 2];               // one tile: [column][latitude]
	__shared__ double red[8][8][4];
	__shared__ double colsc[PT_NC];
	const int ct = blockIdx.x, im = blockIdx.y;
	const int m = im * p.mres;
	const int t0 = t.t0[im];
	const int ntt = t.ntb - t0;
	const double wfac = (m > 0) ? p.mpos_inv : 1.0;
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	// pass 1: column maxima; warp w takes field-component w of the tile,
	// lanes consecutive latitudes
	{
		const int fc = ct * 8 + warp;
		double mx[4] = {0.0, 0.0, 0.0, 0.0};
		for (int row = t0 * PB_T + lane; row < t.ntb * PB_T; row += 32) {
			double g[4];
			gvalues(t, p, im, fc, row, wfac, m, g);
			#pragma unroll
			for (int q = 0; q < 4; q++) mx[q] = fmax(mx[q], fabs(g[q]));
		}
		#pragma unroll
		for (int q = 0; q < 4; q++)
			#pragma unroll
			for (int o = 16; o; o >>= 1) mx[q] = fmax(mx[q], __shfl_xor_sync(0xffffffffu, mx[q], o));
		if (lane == 0) {
			#pragma unroll
			for (int q = 0; q < 4; q++) red[0][warp][q] = mx[q];
		}
	}
	__syncthreads();
	if (tid < 32) {
		const int f = tid >> 2, q = tid & 3;
		const double mx = red[0][f][q];
		int e = 0;
		if (mx > 0.0) frexp(mx, &e);
		// column of (field-component f, even/odd q >> 1, re/im q & 1) within the tile
		const int cl = 16 * (f >> 2) + 2 * (f & 3) + (q & 1) + 8 * (q >> 1);
		colsc[cl] = (mx > 0.0) ? ldexp(1.0, -(e + 2)) : 0.0;
		bexp[(long) im * (nct * PT_NC) + ct * PT_NC + cl] = (mx > 0.0) ? e : -2000;
	}
	__syncthreads();
	// pass 2, per kept tile
	for (int tt = 0; tt < ntt; tt++) {
		const int row0 = (t0 + tt) * PB_T;
		for (int e = tid; e < 8 * PB_T; e += 256) {
			const int fl = e / PB_T, rr = e - fl * PB_T;
			double g[4];
			gvalues(t, p, im, ct * 8 + fl, row0 + rr, wfac, m, g);
			#pragma unroll
			for (int q = 0; q < 4; q++) {
				const int cl = 16 * (fl >> 2) + 2 * (fl & 3) + (q & 1) + 8 * (q >> 1);
				vals[cl][rr] = g[q] * colsc[cl];
			}
		}
		__syncthreads();
		{
			const int cl = tid & 31, g = tid >> 5;            // column, 16-latitude group
			double v[16];
			#pragma unroll
			for (int e16 = 0; e16 < 16; e16++) v[e16] = vals[cl][16 * g + e16];
			uint4 w[NS];
			pack16<NS>(v, w);
			uint8_t* blk = bs + ((t.voff[im] + tt) * nct + ct) * (long) L::B_BYTES + (long) g * L::B_GRP;
			#pragma unroll
			for (int j = 0; j < NS; j++) {
				const int n = PT_NC * j + cl;
				*reinterpret_cast<uint4*>(blk + (n >> 3) * 128 + (n & 7) * 16) = w[j];
			}
		}
		__syncthreads();
	}
}

// ---------------------------------------------------------------------------
// The contraction, persistent: one CTA per SM walks the work items w =
// blockIdx.x, blockIdx.x + gridDim.x, ... (consecutive items are the column
// tiles of one (order, tile), so the digit-blocks they share are read from L2).
//   SYNTH:  item = (order im, latitude tile tb, column tile ct), all tiles
//           (those below the polar threshold are written as zeros); blocks =
//           the 128-step blocks from the tile's first nonzero one to the
//           call's last step.
//   ANALYS: item = (order im, 128-step block kb, column tile ct) over the
//           table's step blocks; blocks = the kept latitude tiles whose first
//           nonzero block is at or before kb.
// Roles: warp 0 copies, warp 1 issues the products into one of two tensor-
// memory accumulator buffers (256 columns each), warps 2-5 read the buffer
// of the previous item, combine it in FP64 and store, then release it.
struct PtItem {
	int im, tile, ct;        // order, latitude tile (SYNTH) or step block, first column tile
	int ntl;                 // column tiles of the item (1 .. CT)
	int nb;                  // blocks to contract (0: nothing; the result is zero)
	int first;               // SYNTH: first step block
};

template <int NS, bool SYNTH, int CT = 1>
__device__ __forceinline__ PtItem ptab_item(const PtabRef& t, const LegParams& p, long w, int nct)
{
	PtItem it;
	const int nctp = (nct + CT - 1) / CT;
	it.ct = (int)(w % nctp) * CT;
	it.ntl = min(CT, nct - it.ct);
	const long e = w / nctp;
	if (SYNTH) {
		it.tile = (int)(e % t.ntb);
		it.im = (int)(e / t.ntb);
		const int m = it.im * p.mres;
		const int nk = (p.llim + p.vec_extra - m) / 2 + 1;
		const int nblk = (nk + PB_K - 1) / PB_K;
		const int t0 = t.t0[it.im];
		it.first = (it.tile >= t0) ? t.kf[t.voff[it.im] + it.tile - t0] : nblk;
		it.nb = (it.tile >= t0 && nk > 0) ? max(0, nblk - it.first) : 0;
	} else {
		// order of the global step block e: the last im with koff[im] <= e
		int lo = 0, hi = p.mlim;
		while (lo < hi) {
			const int mid = (lo + hi + 1) >> 1;
			if (t.koff[mid] <= e) lo = mid; else hi = mid - 1;
		}
		it.im = lo;
		it.tile = (int)(e - t.koff[lo]);
		it.first = 0;
		const int m = it.im * p.mres;
		const int nk = (p.llim + p.vec_extra - m) / 2 + 1;
		const int ntt = t.ntb - t.t0[it.im];
		int n = 0;
		if (it.tile * PB_K < nk)
			for (int ttr = 0; ttr < ntt; ttr++) n += (t.kf[t.voff[it.im] + ttr] <= it.tile) ? 1 : 0;
		it.nb = n;
	}
	return it;
}

// b-th block of an item: first digit-block of Y (global index, digit 0) and
// the digit-stack block; ttr_scan carries the analysis scan position
template <int NS, bool SYNTH>
__device__ __forceinline__ void ptab_block(const PtabRef& t, const PtItem& it, int& ttr_scan, long& ablk, long& bblk)
{
	const long nbk = tab_kblocks(t, it.im);
	const long toff = t.toff[it.im], voff = t.voff[it.im];
	if (SYNTH) {
		const int kb = ttr_scan++;               // starts at it.first
		const int ttr = it.tile - t.t0[it.im];
		ablk = toff + (long) ttr * NS * nbk + kb;
		bblk = t.koff[it.im] + kb;
	} else {
		int ttr = ttr_scan;
		while (t.kf[voff + ttr] > it.tile) ttr++;
		ttr_scan = ttr + 1;
		ablk = toff + (long) ttr * NS * nbk + it.tile;
		bblk = voff + ttr;
	}
}

template <int NS, bool SYNTH, int CT>
__global__ void __launch_bounds__(PT_THREADS, 1) ptab_kernel(PtabRef t, LegParams p, const uint8_t* __restrict__ bs,
                                                             const int* __restrict__ bexp, int nct, long nitems, int* err)
{
	using L = PtLayout<NS, CT>;
	constexpr int PT_RA = L::RA;
	extern __shared__ __align__(1024) uint8_t smem_raw[];
	uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
	uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L::BAR_OFF);
	uint64_t* fullA = bars;
	uint64_t* emptyA = bars + PT_RA;
	uint64_t* fullB = bars + 2 * PT_RA;
	uint64_t* emptyB = fullB + 2;
	uint64_t* tfull = emptyB + 2;
	uint64_t* tempty = tfull + 2;
	uint64_t* drain = tempty + 2;
	uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + L::BAR_OFF + 8 * L::NBAR);
	volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + L::BAR_OFF + 8 * L::NBAR + 4);
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

	if (warp == 1) {
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
		             :: "r"(smem_u32(tmem_slot)), "r"(2u * L::ACC_COLS) : "memory");
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
	}
	if (tid == 0) {
		// one arrival per phase, except tempty: one per epilogue warp
		for (int i = 0; i < L::NBAR; i++) mbar_init(&bars[i], (&bars[i] == &tempty[0] || &bars[i] == &tempty[1]) ? 4 : 1);
		*abort_flag = 0;
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	const uint32_t tmem = *tmem_slot;
	const uint32_t sA = smem_u32(smem + L::A_OFF), sB = smem_u32(smem + L::B_OFF);

	if (warp == 0) {
		if (lane == 0) {
			// producer
			bool ok = true;
			long ua = 0, ub = 0;
			int issuedA[PT_RA], issuedB[2] = {0, 0};
			#pragma unroll
			for (int q = 0; q < PT_RA; q++) issuedA[q] = 0;
			for (long w = blockIdx.x; w < nitems && ok; w += gridDim.x) {
				const PtItem it = ptab_item<NS, SYNTH, CT>(t, p, w, nct);
				int scan = it.first;
				for (int b = 0; b < it.nb && ok; b++) {
					long ablk, bblk;
					ptab_block<NS, SYNTH>(t, it, scan, ablk, bblk);
					const int bsl = (int)(ub & 1);
					if (ub >= 2) ok = mbar_wait(&emptyB[bsl], (uint32_t)(((ub >> 1) - 1) & 1), abort_flag);
					if (!ok) break;
					// the stacks of the item's column tiles are adjacent (column tile fastest)
					mbar_expect_tx(&fullB[bsl], it.ntl * L::B_BYTES);
					bulk_g2s(sB + bsl * L::B_SLOT, bs + (bblk * nct + it.ct) * (long) L::B_BYTES, it.ntl * L::B_BYTES,
					         &fullB[bsl]);
					issuedB[bsl]++;
					ub++;
					const long nbk = tab_kblocks(t, it.im);
					for (int i = 0; i < NS && ok; i++) {
						const int slot = (int)(ua % PT_RA);
						if (ua >= PT_RA) ok = mbar_wait(&emptyA[slot], (uint32_t)(((ua / PT_RA) - 1) & 1), abort_flag);
						if (!ok) break;
						mbar_expect_tx(&fullA[slot], PB_BYTES);
						bulk_g2s(sA + slot * PB_BYTES, t.tab + (ablk + (long) i * nbk) * PB_BYTES, PB_BYTES, &fullA[slot]);
						#pragma unroll
						for (int q = 0; q < PT_RA; q++) if (q == slot) issuedA[q]++;
						ua++;
					}
				}
			}
			// only the last copy into each slot can still be in flight: wait
			// (bounded) for it so that no copy lands after the CTA has left
			#pragma unroll
			for (int q = 0; q < PT_RA; q++) if (issuedA[q]) mbar_wait_quiet(&fullA[q], (issuedA[q] - 1) & 1);
			#pragma unroll
			for (int q = 0; q < 2; q++) if (issuedB[q]) mbar_wait_quiet(&fullB[q], (issuedB[q] - 1) & 1);
		}
	} else if (warp == 1) {
		if (lane == 0) {
			// tensor-core issue
			bool ok = true, any = false;
			long ua = 0, ub = 0, ni = 0;
			for (long w = blockIdx.x; w < nitems && ok; w += gridDim.x) {
				const PtItem it = ptab_item<NS, SYNTH, CT>(t, p, w, nct);
				if (it.nb == 0) continue;
				// CT = 1: alternate between the two buffers; CT = 2: the one buffer
				const int buf = (CT == 1) ? (int)(ni & 1) : 0;
				if (CT == 1 && ni >= 2) ok = mbar_wait(&tempty[buf], (uint32_t)(((ni >> 1) - 1) & 1), abort_flag);
				if (CT == 2 && ni >= 1) ok = mbar_wait(&tempty[0], (uint32_t)((ni - 1) & 1), abort_flag);
				if (!ok) break;
				tc_fence_after();
				const uint32_t dbase = tmem + buf * L::ACC_COLS;
				bool first = true;
				for (int b = 0; b < it.nb && ok; b++) {
					const int bsl = (int)(ub & 1);
					ok = mbar_wait(&fullB[bsl], (uint32_t)((ub >> 1) & 1), abort_flag);
					for (int i = 0; i < NS && ok; i++) {
						const int slot = (int)(ua % PT_RA);
						ok = mbar_wait(&fullA[slot], (uint32_t)((ua / PT_RA) & 1), abort_flag);
						if (!ok) break;
						tc_fence_after();
						const uint32_t idesc = idesc_i8(128, PT_NC * (NS - i), SYNTH ? 0 : 1, 0);
						#pragma unroll
						for (int kk = 0; kk < 4; kk++) {
							uint64_t ad;
							if (SYNTH) {
								// A K-major: M = latitudes (8-row groups 128 B apart), K = steps (16-step core matrices 2048 B apart)
								ad = sdesc(sA + slot * PB_BYTES + kk * 2 * 2048, 2048, 128);
							} else {
								// A MN-major: M = steps (16-byte chunks 2048 B apart), K = latitudes (8-row groups 128 B apart)
								ad = sdesc(sA + slot * PB_BYTES + kk * 4 * 128, 128, 2048);
							}
							// B K-major: N = stacked digit rows (8-row groups 128 B apart), K in 16-byte core matrices B_GRP apart
							#pragma unroll
							for (int c = 0; c < CT; c++) {
								if (c >= it.ntl) break;
								const uint64_t bd = sdesc(sB + bsl * L::B_SLOT + c * L::B_BYTES + kk * 2 * L::B_GRP, L::B_GRP, 128);
								mma_i8(dbase + c * L::ACC_COLS + PT_NC * i, ad, bd, idesc, first ? 0u : 1u);
							}
							first = false;
						}
						any = true;
						mma_commit(&emptyA[slot]);
						ua++;
					}
					if (ok) { mma_commit(&emptyB[bsl]); ub++; }
				}
				if (ok) { mma_commit(&tfull[buf]); ni++; }
			}
			if (any) {
				// products still in flight finish before the memory is released
				mma_commit(drain);
				mbar_wait_quiet(drain, 0);
			}
		}
	} else {
		// epilogue: warps 2-5, TMEM lanes 32 (warp % 4) ..
		const int q = warp & 3;
		long ni = 0;
		for (long w = blockIdx.x; w < nitems; w += gridDim.x) {
			const PtItem it = ptab_item<NS, SYNTH, CT>(t, p, w, nct);
			const int m = it.im * p.mres;
			const int r = 32 * q + lane;
			double accs[CT][PT_NC];
			bool val = false;
			if (it.nb > 0) {
				const int buf = (CT == 1) ? (int)(ni & 1) : 0;
				const uint32_t par = (CT == 1) ? (uint32_t)((ni >> 1) & 1) : (uint32_t)(ni & 1);
				bool ok = mbar_wait(&tfull[buf], par, abort_flag);
				ok = __all_sync(0xffffffffu, ok);
				if (!ok) break;
				tc_fence_after();
				#pragma unroll
				for (int ci = 0; ci < CT; ci++) {
					if (ci >= it.ntl) break;
					const uint32_t trow = tmem + buf * L::ACC_COLS + ci * L::ACC_COLS + ((uint32_t)(32 * q) << 16);
					#pragma unroll
					for (int c = 0; c < PT_NC; c++) accs[ci][c] = 0.0;
					#pragma unroll
					for (int s = NS - 1; s >= 0; s--) {
						int v[16];
						#pragma unroll
						for (int h = 0; h < 2; h++) {
							tmem_ld16(trow + PT_NC * s + 16 * h, v);
							#pragma unroll
							for (int c = 0; c < 16; c++) accs[ci][16 * h + c] = fma(accs[ci][16 * h + c], 0.00390625, (double) v[c]);
						}
					}
				}
				tc_fence_before();
				__syncwarp();
				if (lane == 0) mbar_arrive(&tempty[buf]);
				ni++;
				val = true;
			}
			#pragma unroll
			for (int ci = 0; ci < CT; ci++) {
			if (ci >= it.ntl) break;
			const int ct = it.ct + ci;
			const double* acc = accs[ci];
			// column exponents of the tile, staged per warp
			int* be = reinterpret_cast<int*>(smem + L::BE_OFF) + (q * CT + ci) * PT_NC;
			__syncwarp();
			be[lane] = __ldg(bexp + (long) it.im * (nct * PT_NC) + ct * PT_NC + lane);
			__syncwarp();
			if (SYNTH) {
				const int row = it.tile * PB_T + r;
				if (row < p.nlat_2) {
					const int e = t.yexp[(long) it.im * p.nlat_2 + row];
					const bool v = val && row >= p.mt.tm[it.im] && e > -1000;
					const double cx = p.x[row];
					#pragma unroll
					for (int fl = 0; fl < 8; fl++) {
						const int fc = ct * 8 + fl;
						if (fc >= p.nfc) break;
						const int c0 = 16 * (fl >> 2) + 2 * (fl & 3);          // even re; +1 im; +8 odd
						auto col = [&](int cl) {
							const int bc = be[cl];
							return (v && bc > -1000) ? acc[cl] * pow2(e + bc + 4 - 16) : 0.0;
						};
						const double er = col(c0), ei = col(c0 + 1), orr = col(c0 + 8), oi = col(c0 + 9);
						double nr = fma(cx, orr, er), ni2 = fma(cx, oi, ei);
						double sr = fma(-cx, orr, er), si = fma(-cx, oi, ei);
						const bool vec = (p.ctype[fc / p.nf] != 0) && !p.robert;
						if (vec) { const double sv = p.sinv[row]; nr *= sv; ni2 *= sv; sr *= sv; si *= sv; }
						if (p.adjoint) {
							const double sa = p.w[row] * (m > 0 ? p.mpos_inv : 1.0) / (p.nphi * (m > 0 ? 2.0 : 1.0));
							nr *= sa; ni2 *= sa; sr *= sa; si *= sa;
						}
						double2* Ff = p.F + (long) fc * p.fstride + (long) it.im * p.nlat;
						const int rn = p.south_first ? p.nlat - 1 - row : row;
						const int rs = p.nlat - 1 - rn;
						Ff[rn] = make_double2(nr, ni2);
						Ff[rs] = make_double2(sr, si);
					}
				}
			} else {
				const int nk = (p.llim + p.vec_extra - m) / 2 + 1;
				const int k = it.tile * PB_K + r;
				if (k < nk) {
					double* qrow = p.qq + ((long) p.mt.koff[it.im] + k) * p.ncol + ct * PT_NC;
					#pragma unroll
					for (int c = 0; c < PT_NC; c += 2) {
						if (ct * PT_NC + c >= p.ncol) break;
						const int b0 = be[c], b1 = be[c + 1];
						const double a = (val && b0 > -1000) ? acc[c] * pow2(b0 + 2 - 16) : 0.0;
						const double b = (val && b1 > -1000) ? acc[c + 1] * pow2(b1 + 2 - 16) : 0.0;
						*reinterpret_cast<double2*>(qrow + c) = make_double2(a, b);
					}
				}
			}
			}
		}
	}
	tc_fence_before();
	__syncthreads();
	if (tid == 0 && *abort_flag && err) atomicExch(err, 1);
	if (warp == 1) {
		tc_fence_after();
		asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
		             :: "r"(tmem), "r"(2u * L::ACC_COLS) : "memory");
	}
}

bool grow(void** ptr, size_t* cap, size_t bytes, const char* what)
{
	if (*ptr && *cap >= bytes) return true;
	if (*ptr) cudaFree(*ptr);
	*ptr = nullptr; *cap = 0;
	if (cudaMalloc(ptr, bytes) != cudaSuccess) {
		cudaGetLastError();
		shtb_set_error(3, std::string("out of device memory for ") + what);
		return false;
	}
	*cap = bytes;
	return true;
}

PtabRef ptab_ref(shtns_cfg o)
{
	PtabRef t;
	t.tab = static_cast<const uint8_t*>(o->d_ptab);
	t.toff = o->d_ptoff; t.koff = o->d_pkoff; t.voff = o->d_pvoff; t.t0 = o->d_pt0; t.kf = o->d_pkf;
	t.yexp = o->d_yexp;
	t.ntb = (o->nlat_2 + PB_T - 1) / PB_T;
	t.lmax = o->lmax;
	return t;
}

template <int NS>
void build_table(shtns_cfg o, cudaStream_t st)
{
	const PtabRef t = ptab_ref(o);
	dim3 grid(t.ntb, o->mmax + 1);
	ptab_build_kernel<NS><<<grid, PB_T, 0, st>>>(t, o->nlat_2, o->mres, o->ckseg, o->d_x2, o->d_c, o->mt, o->d_ck,
	                                             static_cast<uint8_t*>(o->d_ptab));
	shtb_count_launch();
}

// The digit table of plan o (the original plan of a clone) with ns digits,
// built on first use.
bool ptab_ensure(shtns_cfg o, int ns, cudaStream_t st)
{
	if (o->d_ptab && o->ptab_ns == ns) return true;
	free_ptab(o);
	if (o->mres != 1) { shtb_set_error(1, "split-precision tables need mres = 1"); return false; }
	const int ntb = (o->nlat_2 + PB_T - 1) / PB_T;
	const int nm = o->mmax + 1;
	std::vector<long> toff(nm), koff(nm), voff(nm);
	std::vector<int> t0(nm);
	long nblocks = 0, kb = 0, tv = 0;
	for (int im = 0; im < nm; im++) {
		t0[im] = std::min(o->tm_h[im] / PB_T, ntb);
		const int ntt = ntb - t0[im];
		const int nbk = (o->kmax_h[im] + PB_K - 1) / PB_K;
		toff[im] = nblocks; koff[im] = kb; voff[im] = tv;
		nblocks += (long) ntt * ns * nbk;
		kb += nbk; tv += ntt;
	}
	// exactness of the INT32 accumulators: ns products of at most 2^14 per step or latitude
	const long kmax_all = std::max<long>(o->kmax_h[0], (long) ntb * PB_T);
	if ((double) kmax_all * ns * 16384.0 >= 2147483647.0) {
		shtb_set_error(1, "split-precision table: grid too large for exact accumulation");
		return false;
	}
	const size_t bytes = (size_t) nblocks * PB_BYTES;
	size_t fr = 0, tot = 0;
	cudaMemGetInfo(&fr, &tot);
	if (bytes + ((size_t) 1 << 30) > fr) {
		shtb_set_error(3, "split-precision table needs " + std::to_string(bytes >> 20) + " MiB, " +
		                  std::to_string(fr >> 20) + " MiB free");
		return false;
	}
	bool okm = shtb_cuda_ok(cudaMalloc(&o->d_ptab, bytes), "split-precision table");
	okm = okm && shtb_cuda_ok(cudaMalloc(&o->d_ptoff, sizeof(long) * 3 * nm), "split-precision table offsets");
	okm = okm && shtb_cuda_ok(cudaMalloc(&o->d_pt0, sizeof(int) * nm), "split-precision table offsets");
	okm = okm && shtb_cuda_ok(cudaMalloc(&o->d_pkf, sizeof(int) * std::max<long>(tv, 1)), "split-precision table offsets");
	if (!okm) { free_ptab(o); return false; }
	o->d_pkoff = o->d_ptoff + nm; o->d_pvoff = o->d_ptoff + 2 * nm;
	cudaMemcpy(o->d_ptoff, toff.data(), sizeof(long) * nm, cudaMemcpyHostToDevice);
	cudaMemcpy(o->d_pkoff, koff.data(), sizeof(long) * nm, cudaMemcpyHostToDevice);
	cudaMemcpy(o->d_pvoff, voff.data(), sizeof(long) * nm, cudaMemcpyHostToDevice);
	cudaMemcpy(o->d_pt0, t0.data(), sizeof(int) * nm, cudaMemcpyHostToDevice);
	o->koff_blocks_h = koff;
	o->ptab_bytes = bytes; o->ptab_ns = ns;
	o->ptab_kblocks = kb; o->ptab_ttiles = tv;
	if (!split_row_exponents(o, st)) { free_ptab(o); shtb_set_error(3, "out of device memory for row exponents"); return false; }
	switch (ns) {
		case 3: build_table<3>(o, st); break;
		case 4: build_table<4>(o, st); break;
		case 5: build_table<5>(o, st); break;
		case 6: build_table<6>(o, st); break;
		default: build_table<7>(o, st); break;
	}
	return shtb_cuda_ok(cudaGetLastError(), "split-precision table");
}

// per-call buffers of plan s: digit stacks for nblocks blocks and the column exponents
bool ptab_buffers(shtns_cfg s, int ns, long nblocks, int nct)
{
	const size_t bb = (size_t) ns * PT_NC * 128;
	if (!grow(&s->d_pbs, &s->pbs_cap, bb * (size_t) nblocks * nct, "split-precision digit stacks")) return false;
	const size_t eb = sizeof(int) * (size_t)(s->mmax + 1) * nct * PT_NC;
	return grow(reinterpret_cast<void**>(&s->d_pexp), &s->pexp_cap, eb, "split-precision column exponents");
}

bool split_err_flag(shtns_cfg s, cudaStream_t st)
{
	if (s->d_split_err) return true;
	if (cudaMalloc(&s->d_split_err, sizeof(int)) != cudaSuccess) { cudaGetLastError(); return false; }
	cudaMemsetAsync(s->d_split_err, 0, sizeof(int), st);
	return true;
}

int num_sms()
{
	static int n = 0;
	if (!n) {
		int dev = 0;
		cudaGetDevice(&dev);
		cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
		if (n <= 0) n = 148;
	}
	return n;
}

// nunits: work items per column tile (synthesis: order x latitude tile;
// analysis: the table's step blocks of the call's orders)
template <int NS, bool SYNTH, int CT>
void launch_contract(const PtabRef& t, const LegParams& p, shtns_cfg s, int nct, long nunits, cudaStream_t st)
{
	using L = PtLayout<NS, CT>;
	const size_t smem = L::TOTAL + 1024;
	static bool attr = false;
	if (!attr) {
		cudaFuncSetAttribute(ptab_kernel<NS, SYNTH, CT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
		attr = true;
	}
	const long nitems = nunits * ((nct + CT - 1) / CT);
	const int grid = (int) std::max<long>(1, std::min<long>(nitems, num_sms()));
	ptab_kernel<NS, SYNTH, CT><<<grid, PT_THREADS, smem, st>>>(t, p, static_cast<const uint8_t*>(s->d_pbs), s->d_pexp, nct,
	                                                           nitems, s->d_split_err);
	shtb_count_launch();
}

// Two column tiles per work item for the analysis (with at least two
// tiles): one read of each table block serves both, which saves more than
// the epilogue, no longer overlapped with the next item's products, costs.
// Measured with 7 digits: lmax 4095, 16 fields 24.3 -> 22.7 ms; lmax 511,
// 64 fields qst (24 tiles) 1.748 -> 1.687 ms.  The synthesis did not gain
// (lmax 4095, 16 fields: 25.4 vs 26.0 ms, within run-to-run noise), so it
// keeps one tile per item.
template <int NS, bool SYNTH>
void contract(const PtabRef& t, const LegParams& p, shtns_cfg s, int nct, long nunits, cudaStream_t st)
{
	if constexpr (!SYNTH) {
		if (nct >= 2) { launch_contract<NS, SYNTH, 2>(t, p, s, nct, nunits, st); return; }
	}
	launch_contract<NS, SYNTH, 1>(t, p, s, nct, nunits, st);
}

template <int NS>
void synth_ns(shtns_cfg s, shtns_cfg o, const LegParams& p, int nct, cudaStream_t st)
{
	const PtabRef t = ptab_ref(o);
	ptab_qslice_kernel<NS><<<dim3(nct, p.mlim + 1), 256, 0, st>>>(t, p.qq, p.ncol, p.mt, p.llim, p.vec_extra, p.mres, nct,
	                                                             static_cast<uint8_t*>(s->d_pbs), s->d_pexp);
	shtb_count_launch();
	contract<NS, true>(t, p, s, nct, (long)(p.mlim + 1) * t.ntb, st);
}

template <int NS>
void analys_ns(shtns_cfg s, shtns_cfg o, const LegParams& p, int nct, cudaStream_t st)
{
	const PtabRef t = ptab_ref(o);
	ptab_gslice_kernel<NS><<<dim3(nct, p.mlim + 1), 256, 0, st>>>(t, p, nct, static_cast<uint8_t*>(s->d_pbs), s->d_pexp);
	shtb_count_launch();
	// step blocks of the orders 0 .. mlim in the table
	const long nkb = (p.mlim < o->mmax) ? o->koff_blocks_h[p.mlim + 1] : o->ptab_kblocks;
	contract<NS, false>(t, p, s, nct, nkb, st);
}

bool ptab_check(const LegParams& p)
{
	if (p.rb.n || p.im0) { shtb_set_error(1, "split precision runs whole transforms on the plain Fourier buffer only"); return false; }
	return true;
}

} // namespace

void launch_ptab_synth(shtns_cfg s, const LegParams& p, cudaStream_t st)
{
	if (!ptab_check(p)) return;
	shtns_cfg o = s->is_clone ? s->base : s;
	const int ns = s->split_ns;
	if (!ptab_ensure(o, ns, st) || !split_err_flag(s, st)) return;
	const int nct = (p.ncol + PT_NC - 1) / PT_NC;
	if (!ptab_buffers(s, ns, o->ptab_kblocks, nct)) return;
	switch (ns) {
		case 3: synth_ns<3>(s, o, p, nct, st); break;
		case 4: synth_ns<4>(s, o, p, nct, st); break;
		case 5: synth_ns<5>(s, o, p, nct, st); break;
		case 6: synth_ns<6>(s, o, p, nct, st); break;
		default: synth_ns<7>(s, o, p, nct, st); break;
	}
}

void launch_ptab_analys(shtns_cfg s, const LegParams& p, cudaStream_t st)
{
	if (!ptab_check(p)) return;
	shtns_cfg o = s->is_clone ? s->base : s;
	const int ns = s->split_ns;
	if (!ptab_ensure(o, ns, st) || !split_err_flag(s, st)) return;
	const int nct = (p.ncol + PT_NC - 1) / PT_NC;
	if (!ptab_buffers(s, ns, o->ptab_ttiles, nct)) return;
	switch (ns) {
		case 3: analys_ns<3>(s, o, p, nct, st); break;
		case 4: analys_ns<4>(s, o, p, nct, st); break;
		case 5: analys_ns<5>(s, o, p, nct, st); break;
		case 6: analys_ns<6>(s, o, p, nct, st); break;
		default: analys_ns<7>(s, o, p, nct, st); break;
	}
}

void free_ptab(shtns_cfg s)
{
	if (!s->is_clone) {
		void* ptrs[] = {s->d_ptab, s->d_ptoff, s->d_pt0, s->d_pkf};
		for (void* q : ptrs) if (q) cudaFree(q);
	}
	s->d_ptab = nullptr; s->ptab_bytes = 0; s->ptab_ns = 0;
	s->d_ptoff = s->d_pkoff = s->d_pvoff = nullptr; s->d_pt0 = nullptr; s->d_pkf = nullptr;
	s->ptab_kblocks = 0; s->ptab_ttiles = 0;
	s->koff_blocks_h.clear();
	if (s->d_pbs) cudaFree(s->d_pbs);
	if (s->d_pexp) cudaFree(s->d_pexp);
	s->d_pbs = nullptr; s->pbs_cap = 0; s->d_pexp = nullptr; s->pexp_cap = 0;
}

extern "C" size_t shtns_b200_split_table_bytes(shtns_cfg s)
{
	if (!s) return 0;
	const shtns_cfg o = s->is_clone ? s->base : s;
	return o->d_ptab ? o->ptab_bytes : 0;
}
