// FP64 Legendre synthesis from a precomputed table of Legendre values.
//
// The on-the-fly kernels (sht_legendre.cu) regenerate Y_k(theta) for every
// tile with the recurrence and stage both GEMM operands through registers.
// On B200 the FP64 tensor-core MMA (mma.sync f64) and the plain FP64
// arithmetic of that staging run on one shared FP64 datapath: while MMAs are
// queued, the staging's dependent FMAs wait behind them (measured: warps doing
// independent FMAs beside MMA warps get under 5 % of their stand-alone rate),
// so the staging of one CTA cannot hide behind the MMAs of the others.
//
// This form removes all arithmetic from the staging.  The values Y_k(theta)
// of every order are computed once per plan into a table, with the same
// operations as the on-the-fly generators (the recurrence from the same
// checkpoints), and each contraction chunk is brought into shared memory by
// bulk copies (cp.async.bulk, no multicast): two 32-step x 32-latitude blocks
// of the table (A) and 32 coefficient rows of 64 columns (B).  One copy warp
// feeds a ring of two stages through mbarriers; four MMA warps with 32 x 32
// warp tiles (eight independent accumulator chains each) issue, per output,
// the MMA sequence of leg_synth_tile (m16n8k4, the same fragment pairs, the
// same k order), so the results are bit-identical to the on-the-fly kernels.
// Three CTAs share an SM.  The CTAs are persistent: each takes every
// gridDim-th work item (order, 64-latitude tile, 64-column tile), heavy
// orders first, and the copy warp runs ahead across item boundaries.
// Measured at lmax 511, 64 fields qst (768 GEMM columns): 1.215 ms against
// 1.32 ms on the fly; 32 x 16 tiles with eight MMA warps and three stages
// (two CTAs per SM) 1.27 ms, 32 x 64 tiles 1.68 ms (registers).
//
// Table layout: per order im, the 32-latitude blocks from the first one kept
// by the polar threshold (tb0) to the equator, each holding the 32-step
// blocks up to step (lmax + 1 - m) / 2 as 32 rows (steps) x 36 doubles
// (latitudes, padded so that fragment loads are free of bank conflicts).
// Block (im, latitude block b, step block kc) is at toff[im] + (b - tb0) nkb
// + kc.  The reference computes these sums in FP64 on the CPU with the values
// generated on the fly (SHT/kernel_SH_to_spat.gen.c:388-409); the table is a
// memory-for-arithmetic choice of this implementation, used within a memory
// budget (option 10).
//
// Every mbarrier wait is bounded (about one second by %globaltimer); a wait
// that gives up records an error flag (shtns_b200_kernel_errors), and the
// copy warp waits (bounded) for the copies it issued before the CTA leaves.
#include "sht_internal.h"
#include "sht_ptx.h"

#include <algorithm>
#include <string>
#include <type_traits>
#include <vector>

namespace {

using namespace shtb_ptx;

constexpr int FT_B = 32;                               // steps and latitudes per table block
constexpr int FT_LD = 36;                              // block row stride in doubles (4 mod 16)
constexpr int FT_BLK = FT_B * FT_LD;                   // doubles per block
constexpr int FT_BLK_BYTES = FT_BLK * 8;
constexpr int FT_BN = 64;                              // GEMM columns per tile
constexpr int FT_BLD = FT_BN + 4;                      // B row stride in doubles (4 mod 16)
constexpr int FT_BROW_BYTES = FT_BLD * 8;
constexpr int FT_STAGE = 2 * FT_BLK_BYTES + FT_B * FT_BROW_BYTES;
static_assert(FT_STAGE % 16 == 0 && FT_BROW_BYTES % 16 == 0, "bulk copy alignment");

struct FtabRef {
	const double* tab;
	const long* toff;        // per order: first block
	const int* tb0;          // per order: first 32-latitude block kept
	const double* zero;      // FT_BN zeros: B rows beyond the call's last step
	int ntb;                 // 32-latitude blocks of the grid
	int lmax;                // table steps of order m: (lmax + 1 - m) / 2 + 1
};

__host__ __device__ __forceinline__ int ft_steps(int lmax, int m) { return (lmax + 1 - m) / 2 + 1; }
__host__ __device__ __forceinline__ int ft_kblocks(int lmax, int m) { return (ft_steps(lmax, m) + FT_B - 1) / FT_B; }

__device__ __forceinline__ void dmma16(double (&c0)[2], double (&c1)[2], double a0, double a1, double b)
{
	asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
	             : "+d"(c0[0]), "+d"(c0[1]), "+d"(c1[0]), "+d"(c1[1]) : "d"(a0), "d"(a1), "d"(b));
}

// ---------------------------------------------------------------------------
// Table build: one warp per (32-latitude block, order), lane = latitude.  The
// segment-wise recurrence of the on-the-fly generators: (Y_{s seg},
// Y_{s seg + 1}) from the checkpoint, then Y_{k} = (c_{2k-1} x^2 + c_{2k-2})
// Y_{k-1} + Y_{k-2} within the segment.
__global__ void __launch_bounds__(32) ftab_build_kernel(FtabRef t, int nlat_2, int mres, int seg,
                                                        const double* __restrict__ x2g, const double* __restrict__ c,
                                                        MTables mt, const double2* __restrict__ ck, double* __restrict__ tab)
{
	const int tb = blockIdx.x, im = blockIdx.y;
	const int tb0 = t.tb0[im];
	if (tb < tb0) return;
	const int m = im * mres;
	const int nkt = ft_steps(t.lmax, m);
	const int nkb = ft_kblocks(t.lmax, m);
	const int r = threadIdx.x, row = tb * FT_B + r;
	const bool live = row < nlat_2;
	const double x2 = live ? x2g[row] : 0.0;
	const double* cc = c + mt.coff[im];
	const double2* ckm = ck + (long)mt.ckoff[im] * nlat_2 + (live ? row : 0);
	double* out = tab + (t.toff[im] + (long)(tb - tb0) * nkb) * FT_BLK;
	double y0 = 0.0, y1 = 0.0;
	for (int k = 0; k < nkb * FT_B; k++) {
		double y = 0.0;
		if (live && k < nkt) {
			const int j = k % seg;
			if (j == 0) {
				const double2 q = ckm[(long)(k / seg) * nlat_2];
				y0 = q.x; y1 = q.y;
				y = y0;
			} else if (j == 1) {
				y = y1;
			} else {
				const double a = fma(cc[2 * k - 1], x2, cc[2 * k - 2]);
				const double y2 = fma(a, y1, y0);
				y0 = y1; y1 = y2;
				y = y2;
			}
		}
		double* o = out + (long)(k / FT_B) * FT_BLK + (k % FT_B) * FT_LD;
		o[r] = y;
		if (r < FT_LD - FT_B) o[FT_B + r] = 0.0;
	}
}

// ---------------------------------------------------------------------------
// Synthesis: item w = (order p.im0 + w / (ntile nnb), 64-latitude tile, 64-column
// tile), column tile fastest.  Warps 0-7: 2 (latitudes) x 4 (columns) MMA
// warps as in leg_synth_tile; warp 8: copies.
// WC: columns per MMA warp (16: 8 MMA warps of 32 x 16; 32: 4 MMA warps of
// 32 x 32), NS: stages of the copy ring, MINB: CTAs per SM.
template <int WC, int NS>
struct FtShape {
	static constexpr int NWN = FT_BN / WC;               // MMA warps along the columns
	static constexpr int NMW = 2 * NWN;                  // MMA warps
	static constexpr int NJ = WC / 8;                    // 8-column fragments per warp
	static constexpr int THREADS = 32 * (NMW + 1);
	static constexpr int BAR_OFF = NS * FT_STAGE;
	static constexpr int SMEM = BAR_OFF + 16 * NS + 16;
};

template <int WC, int NS, int MINB, bool RB>
__global__ void __launch_bounds__(FtShape<WC, NS>::THREADS, MINB)
ftab_synth_kernel(FtabRef t, LegParams p, int ntile, int nnb, long nitems, int* err)
{
	using S = FtShape<WC, NS>;
	constexpr int FT_NS = NS, FT_MMA_WARPS = S::NMW, NJM = S::NJ;
	extern __shared__ __align__(128) uint8_t smem[];
	uint64_t* full = reinterpret_cast<uint64_t*>(smem + S::BAR_OFF);
	uint64_t* empty = full + FT_NS;
	volatile int* abort_flag = reinterpret_cast<volatile int*>(empty + FT_NS);
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	if (tid == 0) {
		for (int i = 0; i < FT_NS; i++) { mbar_init(&full[i], 1); mbar_init(&empty[i], FT_MMA_WARPS); }
		*abort_flag = 0;
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	__syncthreads();
	const uint32_t s0 = smem_u32(smem);
	auto item = [&](long w, int& im, int& tb, int& nb) {
		nb = (int)(w % nnb);
		const long e = w / nnb;
		tb = (int)(e % ntile);
		im = p.im0 + (int)(e / ntile);
	};
	// chunks of an item: none when the whole tile lies above the polar threshold
	auto chunks = [&](int im, int tb) {
		const int nk = (p.llim + p.vec_extra - im * p.mres) / 2 + 1;
		return (tb * 64 + 64 > p.mt.tm[im] && nk > 0) ? (nk + FT_B - 1) / FT_B : 0;
	};

	if (warp == FT_MMA_WARPS) {
		// ---- copy warp ----
		long u = 0;
		int issued[FT_NS];
		#pragma unroll
		for (int q = 0; q < FT_NS; q++) issued[q] = 0;
		bool ok = true;
		for (long w = blockIdx.x; w < nitems && ok; w += gridDim.x) {
			int im, tb, nb;
			item(w, im, tb, nb);
			const int nkc = chunks(im, tb);
			if (nkc == 0) continue;
			const int m = im * p.mres;
			const int nk = (p.llim + p.vec_extra - m) / 2 + 1;
			const int tb0 = t.tb0[im];
			const int nkb = ft_kblocks(t.lmax, m);
			const long tbase = t.toff[im];
			const int c0 = nb * FT_BN;
			const uint32_t row_bytes = (uint32_t)(min(FT_BN, p.ncol - c0) * 8);
			const double* qbase = p.qq + (long)p.mt.koff[im] * p.ncol + c0;
			// latitude blocks of the tile held by the table (the others lie above
			// the polar threshold or beyond the equator: their MMAs are skipped)
			const int b0 = 2 * tb, b1 = 2 * tb + 1;
			const bool v0 = b0 >= tb0 && b0 < t.ntb, v1 = b1 >= tb0 && b1 < t.ntb;
			const uint32_t bytes = (v0 ? FT_BLK_BYTES : 0) + (v1 ? FT_BLK_BYTES : 0) + FT_B * row_bytes;
			for (int kc = 0; kc < nkc; kc++, u++) {
				const int st = (int)(u % FT_NS);
				bool okw = true;
				if (lane == 0 && u >= FT_NS) okw = mbar_wait(&empty[st], (uint32_t)(((u / FT_NS) - 1) & 1), abort_flag);
				if (!__shfl_sync(0xffffffffu, okw, 0)) { ok = false; break; }
				const uint32_t sa = s0 + st * FT_STAGE, sb = sa + 2 * FT_BLK_BYTES;
				if (lane == 0) {
					mbar_expect_tx(&full[st], bytes);
					if (v0) bulk_g2s(sa, t.tab + (tbase + (long)(b0 - tb0) * nkb + kc) * FT_BLK, FT_BLK_BYTES, &full[st]);
					if (v1) bulk_g2s(sa + FT_BLK_BYTES, t.tab + (tbase + (long)(b1 - tb0) * nkb + kc) * FT_BLK, FT_BLK_BYTES,
					                 &full[st]);
					#pragma unroll
					for (int q = 0; q < FT_NS; q++) if (q == st) issued[q]++;
				}
				__syncwarp();
				// one coefficient row per lane; rows at or beyond nk are zeros
				const int k = kc * FT_B + lane;
				const void* src = (k < nk) ? static_cast<const void*>(qbase + (long)k * p.ncol) : static_cast<const void*>(t.zero);
				bulk_g2s(sb + lane * FT_BROW_BYTES, src, row_bytes, &full[st]);
			}
		}
		// the last copies into each stage may still be in flight: wait (bounded)
		// for them so that none lands after the CTA has left
		if (lane == 0) {
			#pragma unroll
			for (int q = 0; q < FT_NS; q++) if (issued[q]) mbar_wait_quiet(&full[q], (uint32_t)((issued[q] - 1) & 1));
		}
	} else {
		// ---- MMA warps ----
		const int wm = warp / S::NWN, wn = warp % S::NWN;
		long u = 0;
		for (long w = blockIdx.x; w < nitems; w += gridDim.x) {
			int im, tb, nb;
			item(w, im, tb, nb);
			const int m = im * p.mres;
			const int nk = (p.llim + p.vec_extra - m) / 2 + 1;
			const int tmm = p.mt.tm[im];
			const int t0 = tb * 64, c0 = nb * FT_BN;
			const int nkc = chunks(im, tb);
			double acc[4][NJM][2];
			#pragma unroll
			for (int i = 0; i < 4; i++)
				#pragma unroll
				for (int j = 0; j < NJM; j++) { acc[i][j][0] = 0.0; acc[i][j][1] = 0.0; }
			// 8 x 8 fragments of this warp that carry results (as leg_synth_tile);
			// the column count is a multiple of 16, so cj1 is even (0, 2, .. NJM)
			const int wr = t0 + wm * 32, wc = c0 + wn * WC;
			const int ri0 = min(4, max(0, (tmm - wr) / 8));
			const int ri1 = min(4, max(0, (p.nlat_2 - wr + 7) / 8));
			const int cj1 = min(NJM, max(0, (p.ncol - wc + 7) / 8));
			const bool p0 = ri0 <= 1 && ri1 > 0, p1 = ri0 <= 3 && ri1 > 2;
			bool ok = true;
			for (int kc = 0; kc < nkc; kc++, u++) {
				const int st = (int)(u % FT_NS);
				ok = __all_sync(0xffffffffu, mbar_wait(&full[st], (uint32_t)((u / FT_NS) & 1), abort_flag));
				if (!ok) break;
				const double* As = reinterpret_cast<const double*>(smem + st * FT_STAGE) + wm * FT_BLK;
				const double* Bs = reinterpret_cast<const double*>(smem + st * FT_STAGE + 2 * FT_BLK_BYTES);
				const int kv = nk - kc * FT_B;
				auto mma_chunk = [&](auto P0, auto P1, auto NJ) {
					#pragma unroll
					for (int kk = 0; kk < FT_B; kk += 4) {
						if (kk >= kv) break;
						const int r = (kk + (lane & 3));
						double a[4], b[NJM];
						#pragma unroll
						for (int i = 0; i < 4; i++)
							if ((i < 2 && P0.value) || (i >= 2 && P1.value)) a[i] = As[r * FT_LD + i * 8 + (lane >> 2)];
						#pragma unroll
						for (int j = 0; j < NJ.value; j++) b[j] = Bs[r * FT_BLD + wn * WC + j * 8 + (lane >> 2)];
						#pragma unroll
						for (int j = 0; j < NJ.value; j++) {
							if constexpr (P0.value) dmma16(acc[0][j], acc[1][j], a[0], a[1], b[j]);
							if constexpr (P1.value) dmma16(acc[2][j], acc[3][j], a[2], a[3], b[j]);
						}
					}
				};
				using T = std::true_type;
				using F = std::false_type;
				auto rows = [&](auto J) {
					if (p0 && p1) mma_chunk(T{}, T{}, J);
					else if (p0) mma_chunk(T{}, F{}, J);
					else if (p1) mma_chunk(F{}, T{}, J);
				};
				switch (cj1) {
					case 2: rows(std::integral_constant<int, 2>{}); break;
					case 4: if constexpr (NJM >= 4) rows(std::integral_constant<int, 4>{}); break;
					case 6: if constexpr (NJM >= 6) rows(std::integral_constant<int, 6>{}); break;
					case 8: if constexpr (NJM >= 8) rows(std::integral_constant<int, 8>{}); break;
					default: break;
				}
				__syncwarp();
				if (lane == 0) mbar_arrive(&empty[st]);
			}
			if (!ok) break;
			// epilogue (as leg_synth_tile): fold hemispheres, 1/sin for vector
			// components, adjoint row weights, store F; each 16-column group of
			// the warp holds 4 field-components (fragment 2g even, 2g + 1 odd)
			#pragma unroll
			for (int g = 0; g < WC / 16; g++) {
				const int fc = ((wc + 16 * g) >> 4) * 4 + (lane & 3);
				if (fc >= p.nfc) continue;
				const bool vec = (p.ctype[fc / p.nf] != 0) && !p.robert;
				double2* Ff = p.F + (long)fc * p.fstride + (long)im * p.nlat;
				#pragma unroll
				for (int i = 0; i < 4; i++) {
					const int tt = t0 + wm * 32 + i * 8 + (lane >> 2);
					if (tt >= p.nlat_2) continue;
					const double cx = p.x[tt];
					const double* ev = acc[i][2 * g];
					const double* od = acc[i][2 * g + 1];
					double nr = fma(cx, od[0], ev[0]), ni = fma(cx, od[1], ev[1]);
					double sr = fma(-cx, od[0], ev[0]), si = fma(-cx, od[1], ev[1]);
					if (tt < tmm) { nr = ni = sr = si = 0.0; }
					if (vec) { const double sv = p.sinv[tt]; nr *= sv; ni *= sv; sr *= sv; si *= sv; }
					if (p.adjoint) {
						const double sa = p.w[tt] * (m > 0 ? p.mpos_inv : 1.0) / (p.nphi * (m > 0 ? 2.0 : 1.0));
						nr *= sa; ni *= sa; sr *= sa; si *= sa;
					}
					const int rn = p.south_first ? p.nlat - 1 - tt : tt;
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
		}
	}
	__syncthreads();
	if (tid == 0 && *abort_flag && err) atomicExch(err, 1);
}

int ft_num_sms()
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

// memory budget of the automatic mode
constexpr size_t FT_AUTO_MAX = (size_t) 8 << 30;

// The table of plan o (the original plan of a clone), built on first use.
// forced: option 10 = 2 (any size that leaves 1 GiB free); otherwise the
// automatic budget (a quarter of the free memory, at most 8 GiB).
bool ftab_ensure(shtns_cfg o, bool forced, cudaStream_t st)
{
	if (o->d_ftab) return true;
	if (o->ftab_failed && !forced) return false;
	// the build allocates and synchronises: not inside a stream capture
	cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
	if (cudaStreamIsCapturing(st, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) return false;
	const int ntb = (o->nlat_2 + FT_B - 1) / FT_B;
	const int nm = o->mmax + 1;
	std::vector<long> toff(nm);
	std::vector<int> tb0(nm);
	long nblocks = 0;
	for (int im = 0; im < nm; im++) {
		tb0[im] = std::min(o->tm_h[im] / FT_B, ntb);
		toff[im] = nblocks;
		nblocks += (long)(ntb - tb0[im]) * ft_kblocks(o->lmax, im * o->mres);
	}
	const size_t bytes = (size_t) nblocks * FT_BLK_BYTES;
	size_t fr = 0, tot = 0;
	cudaMemGetInfo(&fr, &tot);
	const bool fits = forced ? bytes + ((size_t) 1 << 30) <= fr : (bytes <= fr / 4 && bytes <= FT_AUTO_MAX);
	if (!fits) {
		if (forced) shtb_set_error(3, "FP64 Legendre table needs " + std::to_string(bytes >> 20) + " MiB, " +
		                              std::to_string(fr >> 20) + " MiB free");
		o->ftab_failed = 1;
		return false;
	}
	bool okm = cudaMalloc(reinterpret_cast<void**>(&o->d_ftab), bytes) == cudaSuccess;
	okm = okm && cudaMalloc(reinterpret_cast<void**>(&o->d_ftoff), sizeof(long) * nm) == cudaSuccess;
	okm = okm && cudaMalloc(reinterpret_cast<void**>(&o->d_ftb0), sizeof(int) * nm) == cudaSuccess;
	okm = okm && cudaMalloc(reinterpret_cast<void**>(&o->d_fzero), sizeof(double) * FT_BN) == cudaSuccess;
	if (!okm) {
		cudaGetLastError();
		free_ftab(o);
		o->ftab_failed = 1;
		if (forced) shtb_set_error(3, "out of device memory for the FP64 Legendre table");
		return false;
	}
	o->ftab_bytes = bytes;
	cudaMemcpyAsync(o->d_ftoff, toff.data(), sizeof(long) * nm, cudaMemcpyHostToDevice, st);
	cudaMemcpyAsync(o->d_ftb0, tb0.data(), sizeof(int) * nm, cudaMemcpyHostToDevice, st);
	cudaMemsetAsync(o->d_fzero, 0, sizeof(double) * FT_BN, st);
	FtabRef t{o->d_ftab, o->d_ftoff, o->d_ftb0, o->d_fzero, ntb, o->lmax};
	ftab_build_kernel<<<dim3(ntb, nm), 32, 0, st>>>(t, o->nlat_2, o->mres, o->ckseg, o->d_x2, o->d_c, o->mt, o->d_ck,
	                                                o->d_ftab);
	shtb_count_launch();
	// the host vectors are released on return: finish the copies first
	cudaStreamSynchronize(st);
	return shtb_cuda_ok(cudaGetLastError(), "FP64 Legendre table");
}

bool ft_err_flag(shtns_cfg s, cudaStream_t st)
{
	if (s->d_split_err) return true;
	if (cudaMalloc(&s->d_split_err, sizeof(int)) != cudaSuccess) { cudaGetLastError(); return false; }
	cudaMemsetAsync(s->d_split_err, 0, sizeof(int), st);
	return true;
}

} // namespace

// The table form runs the 64 x 64 tile shape (the automatic choice above 32
// GEMM columns, or option 5 = 2) on the plain Fourier buffer; it returns false
// (the caller launches the on-the-fly kernels) when it does not apply or the
// table does not fit the automatic budget.
bool launch_ftab_synth(shtns_cfg s, const LegParams& p, cudaStream_t st)
{
	if (s->ftab_mode == 1 || p.rb.n) return false;
	if (!(p.tile_wm == 2 || (p.tile_wm == 0 && p.ncol > 32))) return false;
	if (leg_simt_selected(p, true)) return false;
	shtns_cfg o = s->is_clone ? s->base : s;
	if (!ftab_ensure(o, s->ftab_mode == 2, st)) return false;
	if (!ft_err_flag(s, st)) return false;
	const int ntile = (p.nlat_2 + 63) / 64;
	const int nnb = (p.ncol + FT_BN - 1) / FT_BN;
	const long nitems = (long)(p.mlim + 1 - p.im0) * ntile * nnb;
	if (nitems <= 0) return true;
	FtabRef t{o->d_ftab, o->d_ftoff, o->d_ftb0, o->d_fzero, (o->nlat_2 + FT_B - 1) / FT_B, o->lmax};
	// 32 x 32 warp tiles, two stages, three CTAs per SM
	constexpr int FT_CFG_WC = 32, FT_CFG_NS = 2, FT_CFG_MINB = 3;
	using SH = FtShape<FT_CFG_WC, FT_CFG_NS>;
	auto kern = ftab_synth_kernel<FT_CFG_WC, FT_CFG_NS, FT_CFG_MINB, false>;
	cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SH::SMEM);
	const int grid = (int) std::min<long>(nitems, (long) FT_CFG_MINB * ft_num_sms());
	kern<<<grid, SH::THREADS, SH::SMEM, st>>>(t, p, ntile, nnb, nitems, s->d_split_err);
	shtb_count_launch();
	return true;
}

void free_ftab(shtns_cfg s)
{
	if (!s->is_clone) {
		void* ptrs[] = {s->d_ftab, s->d_ftoff, s->d_ftb0, s->d_fzero};
		for (void* q : ptrs) if (q) cudaFree(q);
	}
	s->d_ftab = nullptr; s->ftab_bytes = 0; s->d_ftoff = nullptr; s->d_ftb0 = nullptr; s->d_fzero = nullptr;
}
