// Split-precision Legendre synthesis on the FP16 tensor cores (tcgen05).
//
// The FP64 contraction  out[t, c] = sum_k Y_k(t) qq[k, c]  (one order m; t a
// north-hemisphere latitude, c a GEMM column = field-component x {even, odd}
// x {re, im}) is evaluated as an exact sum of products of small integers:
//   Y_k(t) = 2^e_t  sum_i a_i[t,k] 2^(-8(i+1)),  qq[k,c] = 2^f_c sum_j b_j[k,c] 2^(-8(j+1))
// with NS balanced 8-bit slices (|a_0|, |b_0| <= 256, the others <= 130), e_t
// the exponent of max_k |Y_k(t)| (one per row for all k) and f_c that of
// max_k |qq[k,c]|.  Slices are integers, so FP16 holds them exactly, and the
// product of two slices summed over a 128-step window stays below 2^23: each
// FP32 accumulator of one product (i, j) is exact.  Products with
// i + j < NS are kept (the dropped ones weigh 2^(-8 NS) relative to the
// leading one); per window the accumulators of equal i + j are added in FP32
// (still exact: below 2^24) and folded into FP64 registers.  NS = 3..7 keeps
// 24..56 bits; NS <= 5 runs 32 columns per CTA, NS = 6, 7 run 16 (the
// NS (NS + 1) / 2 accumulators of NC columns must fit the 512 tensor-memory
// columns).
//
// Kernel shape (one CTA per order m, 128 latitudes, NC columns; 256 threads):
//   * all threads regenerate Y_k from the recurrence checkpoints in FP64 (row
//     t = tid % 128, 32 steps each), slice them and store the FP16 slices in
//     shared memory in the tensor cores' K-major no-swizzle layout;
//   * the coefficient slices of the chunk (prepared by bslice_kernel) are
//     copied to shared memory next to them;
//   * one thread issues tcgen05.mma (M = 128, N = NC (NS - i), K = 16) for
//     every Y slice i against the stacked coefficient slices j < NS - i,
//     accumulating in tensor memory (NS (NS + 1) / 2 x NC FP32 columns), and
//     commits to an mbarrier; chunks are double-buffered so that the next
//     chunk is generated while the tensor cores work;
//   * every 2 chunks (128 steps) the accumulators are read with tcgen05.ld and
//     added to FP64 registers; the epilogue folds hemispheres and writes F as
//     the FP64 kernel does.
// The reference computes the same sums in FP64 on the CPU
// (kernel_SH_to_spat.gen.c:300-440); this path is a project extension.
#include "sht_internal.h"

#include <cuda_fp16.h>
#include <cstdint>

namespace {

constexpr int SP_M = 128;          // latitudes per CTA = tensor-memory lanes
constexpr int SP_WINK = 128;       // recurrence steps per exact accumulation window
constexpr int SP_THREADS = 256;
constexpr uint64_t SP_WAIT_NS = 1000000000ull;   // time limit of every mbarrier wait

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
	return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ uint64_t global_ns()
{
	uint64_t t;
	asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
	return t;
}

// bounded wait (about one second) for the phase of parity `parity` to
// complete; false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
	const uint32_t a = smem_u32(bar);
	const uint64_t t0 = global_ns();
	for (int it = 0;; it++) {
		if ((it & 1023) == 1023 && global_ns() - t0 > SP_WAIT_NS) return false;
		uint32_t done;
		asm volatile("{\n\t.reg .pred p;\n\t"
		             "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
		             "selp.u32 %0, 1, 0, p;\n\t}"
		             : "=r"(done) : "r"(a), "r"(parity) : "memory");
		if (done) return true;
	}
}

__device__ __forceinline__ void fence_async_smem()
{
	asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// shared-memory matrix descriptor: K-major, no swizzle; lbo / sbo in bytes
// (distance between 8 x 16-byte core matrices along K / along M or N)
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
	uint64_t d = 0;
	d |= (uint64_t)((addr >> 4) & 0x3FFF);
	d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
	d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
	d |= (uint64_t)1 << 46;            // descriptor version of sm_100
	return d;                          // base offset 0, layout type 0 (no swizzle)
}

// instruction descriptor of kind::f16: FP16 x FP16 -> FP32, both K-major
__host__ __device__ constexpr uint32_t idesc_f16(int M, int N)
{
	return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
	asm volatile("{\n\t.reg .pred p;\n\t"
	             "setp.ne.b32 p, %4, 0;\n\t"
	             "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}"
	             :: "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u) : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar)
{
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
	             :: "r"(smem_u32(bar)) : "memory");
}

// 16 consecutive FP32 columns of this warp's 32 lanes
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v)
{
	uint32_t r[16];
	asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
	             "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
	             : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
	               "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
	             : "r"(taddr));
	asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
	#pragma unroll
	for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld4(uint32_t taddr, float* v)
{
	uint32_t r[4];
	asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
	             : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(taddr));
	asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
	#pragma unroll
	for (int i = 0; i < 4; i++) v[i] = __uint_as_float(r[i]);
}

// Balanced 8-bit slices of a value in (-1, 1): x = sum_i a_i 2^(-8(i+1)) up to
// 2^-41.  Two FMAs round x 2^22 and the remainder x 2^18 to integers h, l (the
// magic constant 1.5 2^52 leaves them in the low word); the slices follow by
// integer shifts.  a_0 in [-256, 256], a_1, a_3, a_4 in [-128, 128], a_2 in
// [-130, 130].
__device__ __forceinline__ void slice40(double x, int* a)
{
	const double M52 = 6755399441055744.0;               // 1.5 * 2^52
	const double u0 = fma(x, 4194304.0, M52);             // x 2^22 rounded, + M52
	const int h = __double2loint(u0);
	const double r = fma(x, 4194304.0, M52 - u0);          // exact remainder in [-1/2, 1/2]
	const int l = __double2loint(fma(r, 262144.0, M52));   // remainder 2^18 rounded
	const int a0 = (h + 8192) >> 14;                       // arithmetic shifts: floor division
	const int h1 = h - a0 * 16384;
	const int a1 = (h1 + 32) >> 6;
	const int h2 = h1 - a1 * 64;
	const int R = h2 * 262144 + l;
	const int a2 = (R + 32768) >> 16;
	const int R2 = R - a2 * 65536;
	const int a3 = (R2 + 128) >> 8;
	a[0] = a0; a[1] = a1; a[2] = a2; a[3] = a3; a[4] = R2 - a3 * 256;
}

// Seven balanced 8-bit slices (56 bits): the remainder of the 22 + 18 bits of
// slice40 is rounded once more at 2^-56 (l2, 16 bits).  a_0 in [-256, 256],
// the others in [-130, 130].
__device__ __forceinline__ void slice56(double x, int* a)
{
	const double M52 = 6755399441055744.0;
	const double u0 = fma(x, 4194304.0, M52);
	const int h = __double2loint(u0);
	const double r = fma(x, 4194304.0, M52 - u0);
	const double u1 = fma(r, 262144.0, M52);
	const int l1 = __double2loint(u1);
	const double r1 = fma(r, 262144.0, M52 - u1);
	const int l2 = __double2loint(fma(r1, 65536.0, M52));
	const int a0 = (h + 8192) >> 14;
	const int h1 = h - a0 * 16384;
	const int a1 = (h1 + 32) >> 6;
	const int h2 = h1 - a1 * 64;
	const int R = h2 * 262144 + l1;
	const int a2 = (R + 32768) >> 16;
	const int R2 = R - a2 * 65536;
	const int a3 = (R2 + 128) >> 8;
	const int R3 = R2 - a3 * 256;
	const int T = R3 * 65536 + l2;
	const int a4 = (T + 32768) >> 16;
	const int T2 = T - a4 * 65536;
	const int a5 = (T2 + 128) >> 8;
	a[0] = a0; a[1] = a1; a[2] = a2; a[3] = a3; a[4] = a4; a[5] = a5; a[6] = T2 - a5 * 256;
}

template <int NS>
__device__ __forceinline__ void slice(double x, int* a)
{
	if constexpr (NS <= 5) slice40(x, a);
	else slice56(x, a);
}

// two small integers (|v| < 512) as an FP16 pair, exactly: 1536 + v has
// exponent 10 in FP16, so its bit pattern is 0x6600 + v
__device__ __forceinline__ uint32_t half2_of_ints(int lo, int hi)
{
	const uint32_t bits = (uint32_t)(lo + hi * 65536) + 0x66006600u;
	__half2 v = *reinterpret_cast<const __half2*>(&bits);
	v = __hsub2(v, __halves2half2(__float2half(1536.0f), __float2half(1536.0f)));
	return *reinterpret_cast<uint32_t*>(&v);
}

// Row exponents: e[im][t] with max_k |Y_k(t)| < 2^e (frexp exponent), over
// the steps k < kmax(m) of every order, regenerated from the checkpoints with
// the same operations as the contraction kernels; -2000 when all vanish.
__global__ void yexp_kernel(int nlat_2, int mres, int lmax, int seg, const double* __restrict__ x2g,
                            const double* __restrict__ c, MTables mt, const double2* __restrict__ ck,
                            short* __restrict__ yexp)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	const int im = blockIdx.y;
	if (t >= nlat_2) return;
	const int m = im * mres;
	const int kmax = (lmax + 1 - m) / 2 + 1;
	const double x2 = x2g[t];
	const double* cc = c + mt.coff[im];
	const double2* ckm = ck + (long)mt.ckoff[im] * nlat_2 + t;
	double mx = 0.0;
	for (int ks = 0; ks < kmax; ks += seg) {
		const double2 y = ckm[(long)(ks / seg) * nlat_2];
		double y0 = y.x, y1 = y.y;
		mx = fmax(mx, fabs(y0));
		if (ks + 1 < kmax) mx = fmax(mx, fabs(y1));
		for (int j = 2; j < seg && ks + j < kmax; j++) {
			const int k = ks + j;
			const double a = fma(cc[2 * k - 1], x2, cc[2 * k - 2]);
			const double y2 = fma(a, y1, y0);
			mx = fmax(mx, fabs(y2));
			y0 = y1; y1 = y2;
		}
	}
	int e = -2000;
	if (mx > 0.0) frexp(mx, &e);
	yexp[(long)im * nlat_2 + t] = (short) e;
}

// Coefficient slices.  CTA (column tile ct of NC columns, order im): column
// maxima of qq over the order's steps give f_c (frexp exponent, 0 for an
// all-zero column); then every SP_KC-step chunk of the order is written as NS
// stacked slice matrices (row n = NC j + c, K-major no-swizzle layout of the
// tensor cores: 16-byte groups of 8 steps at (k/8) (NC NS 16) + (n/8) 128 +
// (n%8) 16), zero beyond the order's last step.
template <int NS, int NC, int SP_KC>
__global__ void __launch_bounds__(SP_THREADS) bslice_kernel(const double* __restrict__ qq, int ncol, MTables mt,
                                                            int llim, int vec_extra, int mres, const int* __restrict__ boff,
                                                            int nct, uint4* __restrict__ bsl, int* __restrict__ bexp)
{
	constexpr int NST = NS * NC;                             // stacked rows
	constexpr int BLK = NST * SP_KC * 2 / 16;                // uint4 per chunk block
	__shared__ double red[SP_THREADS / NC][NC];
	__shared__ double colsc[NC];
	const int ct = blockIdx.x, im = blockIdx.y;
	const int m = im * mres;
	const int nk = (llim + vec_extra - m) / 2 + 1;
	const double* qrow = qq + (long)mt.koff[im] * ncol;
	const int tid = threadIdx.x;
	{
		const int cl = tid % NC, kr = tid / NC;
		const int col = ct * NC + cl;
		double mx = 0.0;
		if (col < ncol)
			for (int k = kr; k < nk; k += SP_THREADS / NC) mx = fmax(mx, fabs(qrow[(long)k * ncol + col]));
		red[kr][cl] = mx;
	}
	__syncthreads();
	if (tid < NC) {
		double mx = 0.0;
		for (int r = 0; r < SP_THREADS / NC; r++) mx = fmax(mx, red[r][tid]);
		int e = 0;
		if (mx > 0.0) frexp(mx, &e);
		colsc[tid] = ldexp(1.0, -e);
		bexp[(long)im * (nct * NC) + ct * NC + tid] = e;
	}
	__syncthreads();
	const int nch = (nk + SP_KC - 1) / SP_KC;
	uint4* blk0 = bsl + (long)boff[im] * nct * BLK;
	for (int u = tid; u < nch * NC * (SP_KC / 8); u += SP_THREADS) {
		const int cl = u % NC, g = (u / NC) % (SP_KC / 8), ch = u / (NC * (SP_KC / 8));
		const int col = ct * NC + cl;
		int a[8][NS <= 5 ? 5 : 7];
		#pragma unroll
		for (int e = 0; e < 8; e++) {
			const int k = ch * SP_KC + g * 8 + e;
			const double v = (k < nk && col < ncol) ? qrow[(long)k * ncol + col] * colsc[cl] : 0.0;
			slice<NS>(v, a[e]);
		}
		uint4* blk = blk0 + ((long)ch * nct + ct) * BLK;
		#pragma unroll
		for (int j = 0; j < NS; j++) {
			const int n = j * NC + cl;
			uint4 w;
			w.x = half2_of_ints(a[0][j], a[1][j]);
			w.y = half2_of_ints(a[2][j], a[3][j]);
			w.z = half2_of_ints(a[4][j], a[5][j]);
			w.w = half2_of_ints(a[6][j], a[7][j]);
			blk[(g * (NST * 16) + (n >> 3) * 128 + (n & 7) * 16) / 16] = w;
		}
	}
}

// Shared memory of the contraction kernel (dynamic, 1024-byte aligned):
// A slices [2 buffers][NS][128 x KC FP16], B slices [2][NS x NC x KC FP16],
// two mbarriers, the tensor-memory address and an abort flag.
template <int NS, int NC, int SP_KC>
struct SplitSmem {
	static constexpr int A_BYTES = SP_M * SP_KC * 2;                 // one slice matrix
	static constexpr int B_BYTES = NS * NC * SP_KC * 2;              // stacked coefficient slices
	static constexpr int A_OFF = 0;
	static constexpr int B_OFF = 2 * NS * A_BYTES;
	static constexpr int BAR_OFF = B_OFF + 2 * B_BYTES;
	static constexpr int TOTAL = BAR_OFF + 64;
	static constexpr int ACC_COLS = NC * NS * (NS + 1) / 2;         // FP32 accumulator columns
	static constexpr int TMEM_COLS = ACC_COLS <= 256 ? 256 : 512;
	static_assert(ACC_COLS <= 512, "accumulators exceed tensor memory");
	static_assert(TOTAL + 1024 <= 227 * 1024, "shared memory");
	static constexpr int CPT = NC / 2;                               // columns per thread (8 or 16)
	static __device__ __forceinline__ int acc_col(int i)            // first column of D_i
	{
		return NC * (i * NS - i * (i - 1) / 2);
	}
	// thread group g (0, 1) owns CPT columns: the even (re, im) and odd (re, im)
	// columns of CPT / 4 field-components; local column jl maps to tile column
	static __device__ __forceinline__ int tile_col(int g, int jl)
	{
		const int base = (NC == 32) ? 16 * g : 4 * g;
		return base + (jl < CPT / 2 ? jl : 8 + jl - CPT / 2);
	}
};

template <int NS, int NC, int SP_KC, int SEG>
__global__ void __launch_bounds__(SP_THREADS, 1)
leg_synth_split_kernel(LegParams p, const uint4* __restrict__ bsl, const int* __restrict__ bexp,
                       const int* __restrict__ boff, const short* __restrict__ yexp, int nct, int* __restrict__ err)
{
	using L = SplitSmem<NS, NC, SP_KC>;
	constexpr int CPT = L::CPT;
	constexpr int KH = SP_KC / 2;                            // steps per generator thread and chunk
	constexpr int SP_WIN = SP_WINK / SP_KC;                  // chunks per exact window
	extern __shared__ __align__(1024) uint8_t smem_raw[];
	uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
	uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L::BAR_OFF);
	uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + L::BAR_OFF + 16);
	int* abort_flag = reinterpret_cast<int*>(smem + L::BAR_OFF + 20);

	const int ntb = (p.nlat_2 + SP_M - 1) / SP_M;
	const int tb = blockIdx.x % ntb, ct = blockIdx.x / ntb;
	const int im = blockIdx.y;
	const int m = im * p.mres;
	const int t0 = tb * SP_M;
	const int tid = threadIdx.x, warp = tid >> 5;
	const int nk = (p.llim + p.vec_extra - m) / 2 + 1;
	const int tmm = p.mt.tm[im];
	const int row = tid & (SP_M - 1), half = tid >> 7;      // generator: row, half of a chunk
	const int g = tid >> 7;                                  // read-out: column group
	const int t = t0 + row;
	const bool live = t0 + SP_M > tmm;

	double acc[CPT];
	#pragma unroll
	for (int c = 0; c < CPT; c++) acc[c] = 0.0;
	int erow = -2000;
	if (live) {
		if (warp == 0) {
			asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
			             :: "r"(smem_u32(tmem_slot)), "r"((uint32_t) L::TMEM_COLS) : "memory");
			asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
		}
		if (tid == 0) {
			mbar_init(&bars[0], 1);
			mbar_init(&bars[1], 1);
			*abort_flag = 0;
			asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
		}
		tc_fence_before();
		__syncthreads();
		tc_fence_after();
		const uint32_t tmem = *tmem_slot;

		// generator state: row scale and tables
		const bool grow = t < p.nlat_2;
		if (grow) erow = yexp[(long)im * p.nlat_2 + t];
		const double rsc = (grow && erow > -1000) ? ldexp(1.0, -erow) : 0.0;
		const double x2 = grow ? p.x2[t] : 0.0;
		const double* cm = p.c + p.mt.coff[im];
		const double2* ckm = p.ck + (long)p.mt.ckoff[im] * p.nlat_2 + (grow ? t : 0);
		const uint4* bsrc = bsl + (long)boff[im] * nct * (L::B_BYTES / 16);
		const uint32_t sA = smem_u32(smem + L::A_OFF), sB = smem_u32(smem + L::B_OFF);

		auto generate = [&](int ch, int buf) {
			// Y_k for k = ks..ks+KH-1 of row t, sliced, as 16-byte groups of 8
			// steps; the recurrence starts at the checkpoint at or below ks
			const int ks = ch * SP_KC + KH * half;
			double y0 = 0.0, y1 = 0.0;
			if (rsc != 0.0 && ks < nk) {
				const int kc = (ks / SEG) * SEG;
				const double2 y = __ldg(ckm + (long)(kc / SEG) * p.nlat_2);
				y0 = y.x * rsc; y1 = y.y * rsc;     // scaling by 2^-e commutes with the recurrence
				// advance to (Y_ks, Y_ks+1); Y_ks+1 may lie past the order's last
				// step (coefficient rows are padded to whole 32-step segments)
				for (int k = kc + 2; k <= ks + 1; k++) {
					const double aa = fma(__ldg(cm + 2 * k - 1), x2, __ldg(cm + 2 * k - 2));
					const double y2 = fma(aa, y1, y0);
					y0 = y1; y1 = y2;
				}
			}
			uint8_t* abase = smem + L::A_OFF + buf * NS * L::A_BYTES + (row >> 3) * 128 + (row & 7) * 16;
			#pragma unroll
			for (int q = 0; q < KH / 8; q++) {
				int a[8][NS <= 5 ? 5 : 7];
				#pragma unroll
				for (int e = 0; e < 8; e++) {
					const int j = 8 * q + e;
					double v;
					if (j == 0) v = y0;
					else if (j == 1) v = y1;
					else {
						const int k = ks + j;
						double y2 = 0.0;
						if (k < nk) {
							const double aa = fma(__ldg(cm + 2 * k - 1), x2, __ldg(cm + 2 * k - 2));
							y2 = fma(aa, y1, y0);
						}
						y0 = y1; y1 = y2;
						v = y2;
					}
					if (ks + j >= nk) v = 0.0;
					slice<NS>(v, a[e]);
				}
				const int grp = (KH / 8) * half + q;           // 8-step group within the chunk
				#pragma unroll
				for (int i = 0; i < NS; i++) {
					uint4 w;
					w.x = half2_of_ints(a[0][i], a[1][i]);
					w.y = half2_of_ints(a[2][i], a[3][i]);
					w.z = half2_of_ints(a[4][i], a[5][i]);
					w.w = half2_of_ints(a[6][i], a[7][i]);
					*reinterpret_cast<uint4*>(abase + i * L::A_BYTES + grp * (SP_M * 16)) = w;
				}
			}
			// coefficient slices of the chunk
			const uint4* src = bsrc + ((long)ch * nct + ct) * (L::B_BYTES / 16);
			uint4* dst = reinterpret_cast<uint4*>(smem + L::B_OFF + buf * L::B_BYTES);
			for (int u = tid; u < L::B_BYTES / 16; u += SP_THREADS) dst[u] = __ldg(src + u);
			fence_async_smem();
		};

		auto issue = [&](int buf, bool first) {
			#pragma unroll
			for (int i = 0; i < NS; i++) {
				const uint32_t idesc = idesc_f16(SP_M, NC * (NS - i));
				const uint32_t d = tmem + L::acc_col(i);
				#pragma unroll
				for (int kk = 0; kk < SP_KC / 16; kk++) {
					const uint64_t ad = sdesc(sA + (buf * NS + i) * L::A_BYTES + kk * 2 * (SP_M * 16), SP_M * 16, 128);
					const uint64_t bd = sdesc(sB + buf * L::B_BYTES + kk * 2 * (NS * NC * 16), NS * NC * 16, 128);
					mma_f16(d, ad, bd, idesc, (first && kk == 0) ? 0u : 1u);
				}
			}
			mma_commit(&bars[buf]);
		};

		// window read-out: this warp's 32 lanes, this thread group's CPT columns
		const uint32_t trow = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
		auto readout = [&]() {
			double tq[CPT];
			#pragma unroll
			for (int c = 0; c < CPT; c++) tq[c] = 0.0;
			#pragma unroll
			for (int d = NS - 1; d >= 0; d--) {
				float sd[CPT];
				#pragma unroll
				for (int c = 0; c < CPT; c++) sd[c] = 0.0f;
				#pragma unroll
				for (int i = 0; i <= d; i++) {
					const uint32_t base = trow + L::acc_col(i) + (d - i) * NC;
					float v[CPT];
					if constexpr (NC == 32) {
						tmem_ld16(base + 16 * g, v);
					} else {
						tmem_ld4(base + L::tile_col(g, 0), v);
						tmem_ld4(base + L::tile_col(g, CPT / 2), v + CPT / 2);
					}
					#pragma unroll
					for (int c = 0; c < CPT; c++) sd[c] += v[c];     // exact: integers below 2^24
				}
				#pragma unroll
				for (int c = 0; c < CPT; c++) tq[c] = fma(tq[c], 0.00390625, (double) sd[c]);
			}
			#pragma unroll
			for (int c = 0; c < CPT; c++) acc[c] += tq[c];
			tc_fence_before();
		};

		const int nch = (nk + SP_KC - 1) / SP_KC;
		bool ok = true;
		int issued = 1;
		generate(0, 0);
		__syncthreads();
		if (tid == 0) { tc_fence_after(); issue(0, true); }
		for (int ch = 1; ch < nch && ok; ch++) {
			const int buf = ch & 1;
			if (ch >= 2) ok = __all_sync(0xffffffffu, mbar_wait(&bars[buf], ((ch - 2) >> 1) & 1));   // chunk ch-2 used this buffer
			if (ok) generate(ch, buf);
			const bool first = (ch % SP_WIN) == 0;
			if (ok && first) {
				ok = __all_sync(0xffffffffu, mbar_wait(&bars[buf ^ 1], ((ch - 1) >> 1) & 1));   // window complete
				if (ok) { tc_fence_after(); readout(); }
			}
			if (!ok) atomicExch(abort_flag, 1);
			__syncthreads();
			ok = (*reinterpret_cast<volatile int*>(abort_flag) == 0);
			if (ok) {
				if (tid == 0) { tc_fence_after(); issue(buf, first); }
				issued = ch + 1;
			}
		}
		if (ok) {
			ok = __all_sync(0xffffffffu, mbar_wait(&bars[(nch - 1) & 1], ((nch - 1) >> 1) & 1));
			if (ok) { tc_fence_after(); readout(); }
		}
		if (!ok) {
			// a wait gave up: record it, then give the tensor cores (bounded) time
			// to finish what was issued before the tensor memory is released
			if (err) atomicExch(err, 1);
			mbar_wait(&bars[(issued - 1) & 1], ((issued - 1) >> 1) & 1);
		}
		tc_fence_before();
		__syncthreads();
		if (warp == 0) {
			tc_fence_after();
			asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
			             :: "r"(tmem), "r"((uint32_t) L::TMEM_COLS) : "memory");
		}
	}

	// epilogue: scale, fold hemispheres, store F (as leg_synth_tile)
	if (t >= p.nlat_2) return;
	const double sc = (erow > -1000) ? ldexp(1.0, erow - 16) : 0.0;
	const double cx = p.x[t];
	const int* be = bexp + (long)im * (nct * NC) + ct * NC;
	#pragma unroll
	for (int q = 0; q < CPT / 4; q++) {
		const int c0 = ct * NC + L::tile_col(g, 2 * q);                  // even re column of the field-component
		const int fc = 4 * (c0 >> 4) + ((c0 & 7) >> 1);
		if (fc >= p.nfc) break;
		auto val = [&](int jl) {
			return live ? acc[jl] * sc * ldexp(1.0, be[L::tile_col(g, jl)]) : 0.0;
		};
		const double er = val(2 * q), ei = val(2 * q + 1);
		const double orr = val(CPT / 2 + 2 * q), oi = val(CPT / 2 + 2 * q + 1);
		double nr = fma(cx, orr, er), ni = fma(cx, oi, ei);
		double sr = fma(-cx, orr, er), si = fma(-cx, oi, ei);
		if (t < tmm) { nr = ni = sr = si = 0.0; }
		const bool vec = (p.ctype[fc / p.nf] != 0) && !p.robert;
		if (vec) { const double s = p.sinv[t]; nr *= s; ni *= s; sr *= s; si *= s; }
		if (p.adjoint) {
			const double s = p.w[t] * (m > 0 ? p.mpos_inv : 1.0) / (p.nphi * (m > 0 ? 2.0 : 1.0));
			nr *= s; ni *= s; sr *= s; si *= s;
		}
		double2* Ff = p.F + (long)fc * p.fstride + (long)im * p.nlat;
		const int rn = p.south_first ? p.nlat - 1 - t : t;
		const int rs = p.nlat - 1 - rn;
		Ff[rn] = make_double2(nr, ni);
		Ff[rs] = make_double2(sr, si);
	}
}

} // namespace

// ---------------------------------------------------------------------------
namespace {

template <int NS, int NC, int KC, int SEG>
void launch_split_ns_seg(shtns_cfg s, const LegParams& p, int nct, cudaStream_t st)
{
	using L = SplitSmem<NS, NC, KC>;
	const size_t smem = L::TOTAL + 1024;
	static bool attr = false;
	if (!attr) {
		cudaFuncSetAttribute(leg_synth_split_kernel<NS, NC, KC, SEG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
		attr = true;
	}
	const int ntb = (p.nlat_2 + SP_M - 1) / SP_M;
	bslice_kernel<NS, NC, KC><<<dim3(nct, p.mlim + 1), SP_THREADS, 0, st>>>(
		p.qq, p.ncol, p.mt, p.llim, p.vec_extra, p.mres, s->d_boff, nct,
		static_cast<uint4*>(s->d_bsl), s->d_bexp);
	shtb_count_launch();
	leg_synth_split_kernel<NS, NC, KC, SEG><<<dim3(ntb * nct, p.mlim + 1), SP_THREADS, smem, st>>>(
		p, static_cast<const uint4*>(s->d_bsl), s->d_bexp, s->d_boff, s->d_yexp, nct, s->d_split_err);
	shtb_count_launch();
}

template <int NS, int NC, int KC>
void launch_split_ns(shtns_cfg s, const LegParams& p, cudaStream_t st)
{
	const int nct = (p.ncol + NC - 1) / NC;
	switch (p.ckseg) {
		case 8: launch_split_ns_seg<NS, NC, KC, 8>(s, p, nct, st); break;
		case 16: launch_split_ns_seg<NS, NC, KC, 16>(s, p, nct, st); break;
		default: launch_split_ns_seg<NS, NC, KC, 32>(s, p, nct, st); break;
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

} // namespace

// Tables on first use: row exponents (one pass of the recurrence over every
// order), chunk offsets of the coefficient slices, the error flag.
static bool split_tables(shtns_cfg s, int kc, cudaStream_t st)
{
	if (s->d_boff && s->split_kc != kc) { cudaFree(s->d_boff); s->d_boff = nullptr; }
	if (!s->d_split_err) {
		if (cudaMalloc(&s->d_split_err, sizeof(int)) != cudaSuccess) { cudaGetLastError(); return false; }
		cudaMemsetAsync(s->d_split_err, 0, sizeof(int), st);
	}
	if (!s->d_boff) {
		std::vector<int> boff(s->mmax + 1);
		long tot = 0;
		for (int im = 0; im <= s->mmax; im++) { boff[im] = (int) tot; tot += (s->kmax_h[im] + kc - 1) / kc; }
		if (cudaMalloc(&s->d_boff, sizeof(int) * boff.size()) != cudaSuccess) { cudaGetLastError(); return false; }
		cudaMemcpy(s->d_boff, boff.data(), sizeof(int) * boff.size(), cudaMemcpyHostToDevice);
		s->split_chunks = tot;
		s->split_kc = kc;
	}
	return split_row_exponents(s, st);
}

// Row exponents of the plan (yexp_kernel), computed once on first use.
bool split_row_exponents(shtns_cfg s, cudaStream_t st)
{
	if (!s->d_yexp) {
		if (cudaMalloc(&s->d_yexp, sizeof(short) * (size_t)(s->mmax + 1) * s->nlat_2) != cudaSuccess) {
			cudaGetLastError(); return false;
		}
		dim3 grid((s->nlat_2 + 127) / 128, s->mmax + 1);
		yexp_kernel<<<grid, 128, 0, st>>>(s->nlat_2, s->mres, s->lmax, s->ckseg, s->d_x2, s->d_c, s->mt, s->d_ck, s->d_yexp);
		shtb_count_launch();
	}
	return true;
}

void launch_leg_synth_split(shtns_cfg s, const LegParams& p, cudaStream_t st)
{
	if (s->split_form == 0) { launch_ptab_synth(s, p, st); return; }
	if (p.rb.n) { shtb_set_error(1, "split-precision synthesis writes the plain Fourier buffer only"); return; }
	const int ns = s->split_ns;
	const int nc = ns <= 5 ? 32 : 16;             // accumulators: nc ns (ns + 1) / 2 <= 512 columns
	const int kc = ns <= 6 ? 64 : 32;             // staged steps: two A buffers fit 227 KB
	if (!split_tables(s, kc, st)) { shtb_set_error(3, "out of device memory for split-precision tables"); return; }
	const int nct = (p.ncol + nc - 1) / nc;
	const size_t bsl = (size_t) s->split_chunks * nct * ns * nc * kc * 2;
	const size_t bex = sizeof(int) * (size_t)(s->mmax + 1) * nct * nc;
	if (!grow(&s->d_bsl, &s->bsl_cap, bsl, "coefficient slices")) return;
	if (!grow(reinterpret_cast<void**>(&s->d_bexp), &s->bexp_cap, bex, "column exponents")) return;
	switch (ns) {
		case 3: launch_split_ns<3, 32, 64>(s, p, st); break;
		case 4: launch_split_ns<4, 32, 64>(s, p, st); break;
		case 5: launch_split_ns<5, 32, 64>(s, p, st); break;
		case 6: launch_split_ns<6, 16, 64>(s, p, st); break;
		default: launch_split_ns<7, 16, 32>(s, p, st); break;
	}
}

void free_split(shtns_cfg s)
{
	free_ptab(s);
	void* ptrs[] = {s->d_yexp, s->d_boff, s->d_bsl, s->d_bexp, s->d_split_err};
	for (void* q : ptrs) if (q) cudaFree(q);
	s->d_yexp = nullptr; s->d_boff = nullptr; s->split_chunks = 0; s->split_kc = 0;
	s->d_bsl = nullptr; s->bsl_cap = 0; s->d_bexp = nullptr; s->bexp_cap = 0; s->d_split_err = nullptr;
}

// Waits for the device and returns (and clears) the flags that the
// split-precision kernel and the prefetched FFT kernels set when one of their
// bounded waits gave up.
extern "C" int shtns_b200_kernel_errors(shtns_cfg s)
{
	if (!s) return 0;
	int e = fft_take_wait_error();
	if (!s->d_split_err) return e;
	cudaStreamSynchronize(s->comp_stream);
	int f = 0;
	cudaMemcpy(&f, s->d_split_err, sizeof(int), cudaMemcpyDeviceToHost);
	if (f) cudaMemset(s->d_split_err, 0, sizeof(int));
	return e | f;
}
