// Longitude (phi) FFT stage on sm_100a.
//
// Replaces the reference's FFTW / cuFFT step (sht_init.c:353-518,
// sht_gpu.cu:372-446).  As in the reference, two real latitudes a, b are
// packed into one complex sequence z = v_a + i v_b, so one complex DFT of
// length nphi transforms a latitude pair; the spectra are separated with
// Hermitian symmetry.  A tile is one field-component and 2*S consecutive
// latitudes; its S complex sequences are transformed in shared memory by a
// self-sorting Stockham chain.  Three kernel families:
//   * generic kernels: one tile per CTA, mixed radices (8, 4, 2, 3, 5, 7)
//     chosen at run time, two shared-memory buffers (any supported nphi);
//   * fused kernels (fft3_*): nphi = 3 * 2^k with a compile-time radix chain
//     in one padded in-place buffer, one tile per CTA;
//   * prefetching kernels (fft4_*, the default up to nphi 3072): persistent
//     CTAs that fetch their next tile with tensor copies while the current one
//     is transformed (below).
//
// Synthesis input is F[fc][m][theta] (m <= mlim, exact Fourier coefficients of
// each latitude); output is v(phi_j) = sum_m (2 - delta_m0) Re(F_m e^{i m phi_j}).
// Analysis computes F_m = (1/nphi) sum_j v(phi_j) e^{-i m phi_j}.
// The spatial arrays are theta-contiguous (v[j*nlat + theta]) or
// phi-contiguous (v[theta*nphi + j]).
#include "sht_internal.h"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <algorithm>
#include <atomic>
#include <cstdint>

namespace {

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
	return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
// multiply by sign*i
__device__ __forceinline__ double2 mul_si(double2 a, int sign) { return sign > 0 ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x); }

template <int R> struct Dft;

template <> struct Dft<2> {
	static __device__ __forceinline__ void run(double2* u, int) {
		double2 a = u[0], b = u[1];
		u[0] = cadd(a, b); u[1] = csub(a, b);
	}
};
template <> struct Dft<4> {
	static __device__ __forceinline__ void run(double2* u, int s) {
		double2 t0 = cadd(u[0], u[2]), t1 = csub(u[0], u[2]);
		double2 t2 = cadd(u[1], u[3]), t3 = mul_si(csub(u[1], u[3]), s);
		u[0] = cadd(t0, t2); u[2] = csub(t0, t2);
		u[1] = cadd(t1, t3); u[3] = csub(t1, t3);
	}
};
template <> struct Dft<8> {
	static __device__ __forceinline__ void run(double2* u, int s) {
		const double h = 0.70710678118654752440084436210485;
		// radix-2 split into even / odd halves, each a 4-point DFT
		double2 e[4] = {u[0], u[2], u[4], u[6]};
		double2 o[4] = {u[1], u[3], u[5], u[7]};
		Dft<4>::run(e, s);
		Dft<4>::run(o, s);
		// twiddles w8^q = exp(s*i*pi*q/4)
		double2 o1 = make_double2(h * (o[1].x - s * o[1].y), h * (o[1].y + s * o[1].x));
		double2 o2 = mul_si(o[2], s);
		double2 o3 = make_double2(h * (-o[3].x - s * o[3].y), h * (-o[3].y + s * o[3].x));
		u[0] = cadd(e[0], o[0]); u[4] = csub(e[0], o[0]);
		u[1] = cadd(e[1], o1);   u[5] = csub(e[1], o1);
		u[2] = cadd(e[2], o2);   u[6] = csub(e[2], o2);
		u[3] = cadd(e[3], o3);   u[7] = csub(e[3], o3);
	}
};
template <> struct Dft<3> {
	static __device__ __forceinline__ void run(double2* u, int s) {
		const double c1 = -0.5, s1 = s * 0.86602540378443864676372317075294;
		double2 t = cadd(u[1], u[2]), d = csub(u[1], u[2]);
		double2 mm = make_double2(fma(c1, t.x, u[0].x), fma(c1, t.y, u[0].y));
		u[0] = cadd(u[0], t);
		u[1] = make_double2(mm.x - s1 * d.y, mm.y + s1 * d.x);
		u[2] = make_double2(mm.x + s1 * d.y, mm.y - s1 * d.x);
	}
};
template <> struct Dft<5> {
	static __device__ __forceinline__ void run(double2* u, int s) {
		const double c1 = 0.30901699437494742410229341718282;   // cos(2pi/5)
		const double c2 = -0.80901699437494742410229341718282;  // cos(4pi/5)
		const double s1 = s * 0.95105651629515357211643933337938;  // sin(2pi/5)
		const double s2 = s * 0.58778525229247312916870595463907;  // sin(4pi/5)
		double2 a1 = cadd(u[1], u[4]), b1 = csub(u[1], u[4]);
		double2 a2 = cadd(u[2], u[3]), b2 = csub(u[2], u[3]);
		double2 x0 = u[0];
		u[0] = cadd(x0, cadd(a1, a2));
		double2 r1 = make_double2(x0.x + c1 * a1.x + c2 * a2.x, x0.y + c1 * a1.y + c2 * a2.y);
		double2 r2 = make_double2(x0.x + c2 * a1.x + c1 * a2.x, x0.y + c2 * a1.y + c1 * a2.y);
		// i*(s1 b1 + s2 b2) and i*(s2 b1 - s1 b2)
		double2 i1 = make_double2(-(s1 * b1.y + s2 * b2.y), s1 * b1.x + s2 * b2.x);
		double2 i2 = make_double2(-(s2 * b1.y - s1 * b2.y), s2 * b1.x - s1 * b2.x);
		u[1] = cadd(r1, i1); u[4] = csub(r1, i1);
		u[2] = cadd(r2, i2); u[3] = csub(r2, i2);
	}
};
// 7-point DFT as a direct sum with the roots of unity as literals
// (cos, sin of 2 pi k / 7, symmetric pairs folded).
template <> struct Dft<7> {
	static __device__ __forceinline__ void run(double2* u, int s) {
		const double c[4] = {1.0, 0.62348980185873353053, -0.22252093395631440429, -0.90096886790241912624};
		const double sn[4] = {0.0, 0.78183148246802980871, 0.97492791218182360702, 0.43388373911755812048};
		double2 a[4], b[4];
		#pragma unroll
		for (int q = 1; q < 4; q++) { a[q] = cadd(u[q], u[7 - q]); b[q] = csub(u[q], u[7 - q]); }
		const double2 x0 = u[0];
		u[0] = cadd(x0, cadd(a[1], cadd(a[2], a[3])));
		#pragma unroll
		for (int k = 1; k < 4; k++) {
			double2 r = x0, im = make_double2(0.0, 0.0);
			#pragma unroll
			for (int q = 1; q < 4; q++) {
				const int j = (q * k) % 7;
				const double cq = (j < 4) ? c[j] : c[7 - j];
				const double sq = (j < 4) ? sn[j] : -sn[7 - j];
				r.x = fma(cq, a[q].x, r.x);  r.y = fma(cq, a[q].y, r.y);
				im.x = fma(sq, b[q].x, im.x); im.y = fma(sq, b[q].y, im.y);
			}
			// y_k = r + i s im,  y_{7-k} = r - i s im
			const double2 t = make_double2(-s * im.y, s * im.x);
			u[k] = cadd(r, t);
			u[7 - k] = csub(r, t);
		}
	}
};

// Shared-memory layout: element i of sequence s lives at s*seq + i + i/8.
// The pad of one slot per 8 elements spreads the stride-R writes of the first
// Stockham pass over the banks, and seq = 2 mod 8 (in 16-byte units) spreads
// the S sequences, so both the passes and the latitude-pair loads/stores are
// free of bank conflicts.
__device__ __forceinline__ int sidx(int s, int i, int seq) { return s * seq + i + (i >> 3); }

// q = x / d, r = x % d for 0 <= x < 2^22 with a float reciprocal and one
// correction step (avoids the integer division sequence in the inner loops).
__device__ __forceinline__ void divmod(int x, int d, float inv, int& q, int& r)
{
	q = __float2int_rz(__int2float_rn(x) * inv);
	r = x - q * d;
	if (r < 0) { q--; r += d; }
	else if (r >= d) { q++; r -= d; }
}

// One Stockham pass of radix R over S sequences of length N, from X to Y.
// Butterfly b of a sequence reads element b + q*N/R (q < R), applies twiddles
// w^{q*k*N/(p*R)} with k = b mod p, runs the R-point DFT and writes element
// (b - k)*R + k + q*p.
template <int R>
__device__ __forceinline__ void fft_pass(const double2* __restrict__ X, double2* __restrict__ Y, int N, int S, int seq,
                                         int p, const double2* __restrict__ tw, int sign)
{
	const int nbf = N / R;
	const int total = S * nbf;
	const int tstep = N / (p * R);
	const float inv_nbf = 1.0f / nbf, inv_p = 1.0f / p;
	for (int g = threadIdx.x; g < total; g += blockDim.x) {
		int sq, b, q0, k;
		divmod(g, nbf, inv_nbf, sq, b);
		divmod(b, p, inv_p, q0, k);
		double2 u[R];
		#pragma unroll
		for (int q = 0; q < R; q++) u[q] = X[sidx(sq, b + q * nbf, seq)];
		if (k) {
			// w^q by repeated multiplication from one table entry (error ~q ulp)
			double2 w1 = __ldg(tw + k * tstep);
			if (sign < 0) w1.y = -w1.y;
			double2 w = w1;
			#pragma unroll
			for (int q = 1; q < R; q++) {
				u[q] = cmul(u[q], w);
				if (q + 1 < R) w = cmul(w, w1);
			}
		}
		Dft<R>::run(u, sign);
		const int o = (b - k) * R + k;
		#pragma unroll
		for (int q = 0; q < R; q++) Y[sidx(sq, o + q * p, seq)] = u[q];
	}
	__syncthreads();
}

// Runs all passes; returns the buffer (X or Y) that holds the result.
__device__ __forceinline__ double2* fft_run(double2* X, double2* Y, int N, int S, int seq, unsigned long long rcode,
                                            int nradix, const double2* __restrict__ tw, int sign)
{
	int pp = 1;
	for (int r = 0; r < nradix; r++) {
		const int R = (int)((rcode >> (4 * r)) & 15);
		switch (R) {
			case 8: fft_pass<8>(X, Y, N, S, seq, pp, tw, sign); break;
			case 4: fft_pass<4>(X, Y, N, S, seq, pp, tw, sign); break;
			case 2: fft_pass<2>(X, Y, N, S, seq, pp, tw, sign); break;
			case 3: fft_pass<3>(X, Y, N, S, seq, pp, tw, sign); break;
			case 5: fft_pass<5>(X, Y, N, S, seq, pp, tw, sign); break;
			default: fft_pass<7>(X, Y, N, S, seq, pp, tw, sign); break;
		}
		pp *= R;
		double2* t = X; X = Y; Y = t;
	}
	return X;
}

__device__ __forceinline__ int seq_len(int N, int S)
{
	const int a = N + (N >> 3);
	return a + (((S >= 8 ? 1 : 8 / S) - a) & 7);
}

// Synthesis: F[fc][m][theta] (m <= mlim) -> spatial field-component fc.
// Sequence s of the CTA packs latitudes lat0+2s (real part) and lat0+2s+1
// (imaginary part): Z_k = A_k + i B_k, Z_{N-k} = conj(A_k) + i conj(B_k).
template <int S>
__global__ void __launch_bounds__(768) fft_synth_kernel(FftParams p)
{
	extern __shared__ double2 smem[];
	const int N = p.N, T = blockDim.x, seq = seq_len(N, S);
	double2* X = smem;
	double2* Y = smem + S * seq;
	const int fc = blockIdx.y;
	const int lat0 = blockIdx.x * 2 * S;
	const double2* Ff = p.F + (long)fc * p.fstride;
	const int ml = p.mlim;
	// zero the band between +mlim and -mlim
	const int nz = N - 2 * ml - 1;
	for (int e = threadIdx.x; e < S * nz; e += T) {
		const int s = e / nz, i = ml + 1 + (e - s * nz);
		X[sidx(s, i, seq)] = make_double2(0.0, 0.0);
	}
	const int nload = (ml + 1) * S;
	for (int e0 = threadIdx.x; e0 < nload; e0 += 4 * T) {
		double2 a[4], b[4];
		#pragma unroll
		for (int u = 0; u < 4; u++) {
			const int e = e0 + u * T;
			const int k = e / S, s = e - k * S;
			const int ra = lat0 + 2 * s;
			a[u] = make_double2(0.0, 0.0); b[u] = make_double2(0.0, 0.0);
			if (e < nload && ra < p.nlat) {
				a[u] = __ldg(Ff + (long)k * p.nlat + ra);
				b[u] = __ldg(Ff + (long)k * p.nlat + ra + 1);
			}
		}
		#pragma unroll
		for (int u = 0; u < 4; u++) {
			const int e = e0 + u * T;
			if (e >= nload) continue;
			const int k = e / S, s = e - k * S;
			if (k == 0) { a[u].y = 0.0; b[u].y = 0.0; }
			X[sidx(s, k, seq)] = make_double2(a[u].x - b[u].y, a[u].y + b[u].x);
			if (k > 0) X[sidx(s, N - k, seq)] = make_double2(a[u].x + b[u].y, b[u].x - a[u].y);
		}
	}
	__syncthreads();
	X = fft_run(X, Y, N, S, seq, p.rcode, p.nradix, p.tw, +1);
	const int c = fc / p.nf;
	double* out = (c == 0 ? p.spat[0] : c == 1 ? p.spat[1] : p.spat[2]) + (long)(fc - c * p.nf) * p.spat_dist;
	if (!p.phi_contiguous) {
		for (int e = threadIdx.x; e < N * S; e += T) {
			const int j = e / S, s = e - j * S;
			const int row = lat0 + 2 * s;
			if (row < p.nlat) {
				const double2 z = X[sidx(s, j, seq)];
				double* o = out + (long)j * p.nlat + row;
				if (p.vec2) *reinterpret_cast<double2*>(o) = z;
				else { o[0] = z.x; o[1] = z.y; }
			}
		}
	} else {
		for (int e = threadIdx.x; e < N * S; e += T) {
			const int s = e / N, j = e - s * N;
			const int row = lat0 + 2 * s;
			if (row < p.nlat) {
				const double2 z = X[sidx(s, j, seq)];
				out[(long)row * N + j] = z.x;
				out[(long)(row + 1) * N + j] = z.y;
			}
		}
	}
}

// Analysis: spatial field-component fc -> F[fc][m][theta] = A_m / N for m <= mlim,
// with A_k = (Z_k + conj Z_{N-k})/2 and B_k = (Z_k - conj Z_{N-k})/(2i).
template <int S>
__global__ void __launch_bounds__(768) fft_analys_kernel(FftParams p)
{
	extern __shared__ double2 smem[];
	const int N = p.N, T = blockDim.x, seq = seq_len(N, S);
	double2* X = smem;
	double2* Y = smem + S * seq;
	const int fc = blockIdx.y;
	const int lat0 = blockIdx.x * 2 * S;
	const int c = fc / p.nf;
	const double* in = (c == 0 ? p.spat_in[0] : c == 1 ? p.spat_in[1] : p.spat_in[2]) + (long)(fc - c * p.nf) * p.spat_dist;
	if (!p.phi_contiguous) {
		// 8 independent loads in flight per thread before the shared-memory stores
		for (int e0 = threadIdx.x; e0 < N * S; e0 += 8 * T) {
			double2 v[8];
			#pragma unroll
			for (int u = 0; u < 8; u++) {
				const int e = e0 + u * T;
				const int j = e / S, s = e - j * S;
				const int row = lat0 + 2 * s;
				v[u] = make_double2(0.0, 0.0);
				if (e < N * S && row < p.nlat) {
					const double* i0 = in + (long)j * p.nlat + row;
					v[u] = p.vec2 ? __ldg(reinterpret_cast<const double2*>(i0)) : make_double2(__ldg(i0), __ldg(i0 + 1));
				}
			}
			#pragma unroll
			for (int u = 0; u < 8; u++) {
				const int e = e0 + u * T;
				if (e < N * S) { const int j = e / S, s = e - j * S; X[sidx(s, j, seq)] = v[u]; }
			}
		}
	} else {
		for (int e = threadIdx.x; e < N * S; e += T) {
			const int s = e / N, j = e - s * N;
			const int row = lat0 + 2 * s;
			double2 v = make_double2(0.0, 0.0);
			if (row < p.nlat) v = make_double2(in[(long)row * N + j], in[(long)(row + 1) * N + j]);
			X[sidx(s, j, seq)] = v;
		}
	}
	__syncthreads();
	X = fft_run(X, Y, N, S, seq, p.rcode, p.nradix, p.tw, -1);
	double2* Ff = p.F + (long)fc * p.fstride;
	const double sc = 0.5 / N;
	for (int e = threadIdx.x; e < (p.mlim + 1) * S; e += T) {
		const int k = e / S, s = e - k * S;
		const int ra = lat0 + 2 * s;
		const double2 z = X[sidx(s, k, seq)];
		const double2 w = X[sidx(s, k ? N - k : 0, seq)];
		if (ra < p.nlat) {
			Ff[(long)k * p.nlat + ra] = make_double2(sc * (z.x + w.x), sc * (z.y - w.y));
			Ff[(long)k * p.nlat + ra + 1] = make_double2(sc * (z.y + w.y), -sc * (z.x - w.x));
		}
	}
}

// ===========================================================================
// Fused kernels for nphi = 3 * 2^k (192 ... 6144), the sizes of Gauss grids
// with nphi = 2 nlat = 3 (lmax+1).  The radix sequence is fixed at compile
// time, so every index, stride and twiddle step is a constant.  The first
// pass reads its butterfly inputs straight from global memory (no staging
// copy) and, for synthesis, the last pass writes straight to global memory.
// Intermediate passes work in place in one padded shared buffer: each thread
// loads its butterflies into registers, the block synchronises, then writes.
// Thread g of the block handles sequence g % S and butterfly g / S, so the
// S sequences of a butterfly index are neighbours in a warp (contiguous
// 16-byte latitude pairs in global memory).
template <int... Rs> struct RadixList {};

template <int N> struct NphiPlan;
template <> struct NphiPlan<192>  { using L = RadixList<8, 8, 3>; };
template <> struct NphiPlan<384>  { using L = RadixList<8, 4, 4, 3>; };
template <> struct NphiPlan<768>  { using L = RadixList<8, 8, 4, 3>; };
template <> struct NphiPlan<1536> { using L = RadixList<8, 8, 8, 3>; };
template <> struct NphiPlan<3072> { using L = RadixList<8, 8, 4, 4, 3>; };
template <> struct NphiPlan<6144> { using L = RadixList<8, 8, 8, 4, 3>; };
template <> struct NphiPlan<12288> { using L = RadixList<8, 8, 8, 8, 3>; };
template <> struct NphiPlan<96>  { using L = RadixList<8, 4, 3>; };
template <> struct NphiPlan<128> { using L = RadixList<8, 4, 4>; };

template <int N, int S>
struct Geo {
	static constexpr int A = N + (N >> 3);
	// sequence stride 8/S mod 8 (16-byte units) for S <= 8, 1 mod 8 beyond, so
	// that the 8 lanes of a 16-byte access phase, on consecutive sequences,
	// hit distinct banks
	static constexpr int SEQ = A + (((S >= 8 ? 1 : 8 / S) - A) & 7);
	// one radix-8 butterfly per thread, at most 768 threads (two or more per thread beyond)
	static constexpr int T = (S * N / 8 <= 768) ? S * N / 8 : 768;
	static __device__ __forceinline__ int at(int s, int i) { return s * SEQ + i + (i >> 3); }
};

// twiddle powers u[q] *= w^q, w = exp(sign 2 pi i k step / N)
template <int R>
__device__ __forceinline__ void twiddle(double2* u, const double2* __restrict__ tw, int idx, int sign)
{
	double2 w1 = __ldg(tw + idx);
	if (sign < 0) w1.y = -w1.y;
	double2 w = w1;
	#pragma unroll
	for (int q = 1; q < R; q++) {
		u[q] = cmul(u[q], w);
		if (q + 1 < R) w = cmul(w, w1);
	}
}

// One middle pass (in place in X).  P = product of earlier radices.
// DENSE: the outputs go to X[j * S + s] (rows of S complex values, for a
// tensor store) instead of the padded sequence layout
template <int N, int S, int R, int P, bool DENSE = false>
__device__ __forceinline__ void mid_pass(double2* X, const double2* __restrict__ tw, int sign, int tid)
{
	using G = Geo<N, S>;
	constexpr int NBF = N / R, TOT = S * NBF, NB = (TOT + G::T - 1) / G::T, TSTEP = N / (P * R);
	double2 u[NB][R];
	int dst[NB], ss[NB];
	#pragma unroll
	for (int i = 0; i < NB; i++) {
		const int g = tid + i * G::T;
		dst[i] = -1;
		if (g < TOT) {
			const int s = g % S, b = g / S, k = b % P;
			#pragma unroll
			for (int q = 0; q < R; q++) u[i][q] = X[G::at(s, b + q * NBF)];
			if (P > 1 && k) twiddle<R>(u[i], tw, k * TSTEP, sign);
			Dft<R>::run(u[i], sign);
			dst[i] = (b - k) * R + k;
			ss[i] = s;
		}
	}
	__syncthreads();
	#pragma unroll
	for (int i = 0; i < NB; i++)
		if (dst[i] >= 0) {
			#pragma unroll
			for (int q = 0; q < R; q++) X[DENSE ? (dst[i] + q * P) * S + ss[i] : G::at(ss[i], dst[i] + q * P)] = u[i][q];
		}
	__syncthreads();
}

// Last pass of an analysis chain ending in radix 3 (P = N/3): thread item
// (s, b), b = 0 .. P/2, runs the butterflies b and P - b of sequence s, which
// hold both members of the pairs (z_k, z_{N-k}) for k = b, P - b and P + b
// (b = 0: k = 0, P; b = P/2: k = P/2), and hands each pair to st(s, k, z_k,
// z_{N-k}).  Every k < N/2 is handed over once; no shared-memory output.
template <int N, int S, class Store>
__device__ __forceinline__ void last_pass_pairs(const double2* X, const double2* __restrict__ tw, int sign, Store& st, int tid)
{
	using G = Geo<N, S>;
	constexpr int P = N / 3, H = P / 2, ITEMS = S * (H + 1), NB = (ITEMS + G::T - 1) / G::T;
	#pragma unroll
	for (int i = 0; i < NB; i++) {
		const int g = tid + i * G::T;
		if (g < ITEMS) {
			const int s = g % S, b = g / S;
			double2 u[3];
			#pragma unroll
			for (int q = 0; q < 3; q++) u[q] = X[G::at(s, b + q * P)];
			if (b) twiddle<3>(u, tw, b, sign);
			Dft<3>::run(u, sign);                       // z_{b + q P} = u[q]
			if (b == 0) {
				st(s, 0, u[0], u[0]);
				st(s, P, u[1], u[2]);
			} else if (b == H) {
				st(s, H, u[0], u[2]);
			} else {
				const int bp = P - b;
				double2 v[3];
				#pragma unroll
				for (int q = 0; q < 3; q++) v[q] = X[G::at(s, bp + q * P)];
				twiddle<3>(v, tw, bp, sign);
				Dft<3>::run(v, sign);                   // z_{P - b + q P} = v[q]
				st(s, b, u[0], v[2]);
				st(s, bp, v[0], u[2]);
				st(s, P + b, u[1], v[1]);
			}
		}
	}
}

// Pass chain: first pass from a loader, middle passes in shared memory, last
// pass to shared memory (MODE 0), to a storer (MODE 1), to shared memory in
// rows of S complex values (MODE 2), or as (z_k, z_{N-k}) pairs to a storer
// (MODE 3, last radix 3).
template <int N, int S, int P, int MODE, int R, int... Rest>
struct Chain {
	template <class Store>
	static __device__ __forceinline__ void run(double2* X, const double2* tw, int sign, Store& st, int tid)
	{
		if constexpr (sizeof...(Rest) == 0) {
			if constexpr (MODE == 3) {
				static_assert(R == 3 && P * 3 == N, "the pair pass is the last radix-3 pass");
				last_pass_pairs<N, S>(X, tw, sign, st, tid);
			} else if constexpr (MODE == 1) {
				// last pass: k = b (b < P = N/R), outputs b + q*P go to global memory
				using G = Geo<N, S>;
				constexpr int NBF = N / R, TOT = S * NBF, NB = (TOT + G::T - 1) / G::T, TSTEP = N / (P * R);
				#pragma unroll
				for (int i = 0; i < NB; i++) {
					const int g = tid + i * G::T;
					if (g < TOT) {
						const int s = g % S, b = g / S;
						double2 u[R];
						#pragma unroll
						for (int q = 0; q < R; q++) u[q] = X[G::at(s, b + q * NBF)];
						if (b) twiddle<R>(u, tw, b * TSTEP, sign);
						Dft<R>::run(u, sign);
						#pragma unroll
						for (int q = 0; q < R; q++) st(s, b + q * P, u[q]);
					}
				}
			} else {
				mid_pass<N, S, R, P, MODE == 2>(X, tw, sign, tid);
			}
		} else {
			mid_pass<N, S, R, P>(X, tw, sign, tid);
			Chain<N, S, P * R, MODE, Rest...>::run(X, tw, sign, st, tid);
		}
	}
};

struct NoHook { __device__ __forceinline__ void operator()() const {} };

// after_first() runs once the first pass has written X and the block has
// synchronised (the input is no longer read)
template <int N, int S, int MODE, class Load, class Store, class Hook, int R0, int... Rest>
__device__ __forceinline__ void fused_fft(double2* X, const double2* tw, int sign, Load& ld, Store& st, const Hook& after_first,
                                          int tid, RadixList<R0, Rest...>)
{
	// first pass: butterfly b reads elements b + q*N/R0 from global, no twiddles
	using G = Geo<N, S>;
	constexpr int NBF = N / R0, TOT = S * NBF, NB = (TOT + G::T - 1) / G::T;
	double2 u[NB][R0];
	#pragma unroll
	for (int i = 0; i < NB; i++) {
		const int g = tid + i * G::T;
		if (g < TOT) {
			const int s = g % S, b = g / S;
			#pragma unroll
			for (int q = 0; q < R0; q++) u[i][q] = ld(s, b + q * NBF);
		}
	}
	#pragma unroll
	for (int i = 0; i < NB; i++) {
		const int g = tid + i * G::T;
		if (g < TOT) {
			const int s = g % S, b = g / S;
			Dft<R0>::run(u[i], sign);
			#pragma unroll
			for (int q = 0; q < R0; q++) X[G::at(s, b * R0 + q)] = u[i][q];
		}
	}
	__syncthreads();
	after_first();
	Chain<N, S, R0, MODE, Rest...>::run(X, tw, sign, st, tid);
}

template <int N, int S>
__global__ void __launch_bounds__(Geo<N, S>::T) fft3_synth_kernel(FftParams p)
{
	extern __shared__ double2 smem[];
	const int fc = blockIdx.y;
	const int lat0 = blockIdx.x * 2 * S;
	const double2* __restrict__ Ff = p.F + (long)fc * p.fstride;
	const int ml = p.mlim, nlat = p.nlat;
	auto ld = [&](int s, int j) -> double2 {
		const int ra = lat0 + 2 * s;
		const int k = (j <= ml) ? j : ((j >= N - ml) ? N - j : -1);
		if (k < 0 || ra >= nlat) return make_double2(0.0, 0.0);
		double2 a = __ldg(Ff + (long)k * nlat + ra), b = __ldg(Ff + (long)k * nlat + ra + 1);
		if (k == 0) { a.y = 0.0; b.y = 0.0; }
		return (j <= ml) ? make_double2(a.x - b.y, a.y + b.x) : make_double2(a.x + b.y, b.x - a.y);
	};
	const int c = fc / p.nf;
	double* out = (c == 0 ? p.spat[0] : c == 1 ? p.spat[1] : p.spat[2]) + (long)(fc - c * p.nf) * p.spat_dist;
	const bool phi = p.phi_contiguous, v2 = p.vec2;
	auto st = [&](int s, int j, double2 z) {
		const int row = lat0 + 2 * s;
		if (row >= nlat) return;
		if (!phi) {
			double* o = out + (long)j * nlat + row;
			if (v2) *reinterpret_cast<double2*>(o) = z;
			else { o[0] = z.x; o[1] = z.y; }
		} else {
			out[(long)row * N + j] = z.x;
			out[(long)(row + 1) * N + j] = z.y;
		}
	};
	fused_fft<N, S, true>(smem, p.tw, +1, ld, st, NoHook{}, threadIdx.x, typename NphiPlan<N>::L{});
}

template <int N, int S>
__global__ void __launch_bounds__(Geo<N, S>::T) fft3_analys_kernel(FftParams p)
{
	extern __shared__ double2 smem[];
	const int fc = blockIdx.y;
	const int lat0 = blockIdx.x * 2 * S;
	const int nlat = p.nlat;
	const int c = fc / p.nf;
	const double* in = (c == 0 ? p.spat_in[0] : c == 1 ? p.spat_in[1] : p.spat_in[2]) + (long)(fc - c * p.nf) * p.spat_dist;
	const bool phi = p.phi_contiguous, v2 = p.vec2;
	auto ld = [&](int s, int j) -> double2 {
		const int row = lat0 + 2 * s;
		if (row >= nlat) return make_double2(0.0, 0.0);
		if (!phi) {
			const double* i0 = in + (long)j * nlat + row;
			return v2 ? __ldg(reinterpret_cast<const double2*>(i0)) : make_double2(__ldg(i0), __ldg(i0 + 1));
		}
		return make_double2(__ldg(in + (long)row * N + j), __ldg(in + (long)(row + 1) * N + j));
	};
	// Fourier rows straight from the last radix pass (pairs z_k, z_{N-k})
	double2* Ff = p.F + (long)fc * p.fstride;
	const double sc = 0.5 / N;
	const int ml = p.mlim;
	auto st = [&](int s, int k, double2 z, double2 w) {
		const int ra = lat0 + 2 * s;
		if (k > ml || ra >= nlat) return;
		const double2 fa = make_double2(sc * (z.x + w.x), sc * (z.y - w.y));
		const double2 fb = make_double2(sc * (z.y + w.y), -sc * (z.x - w.x));
		double2* o = Ff + (long)k * nlat + ra;
		if (((uintptr_t) o & 31) == 0)      // one 32-byte store for the latitude pair
			asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};"
			             :: "l"(o), "d"(fa.x), "d"(fa.y), "d"(fb.x), "d"(fb.y) : "memory");
		else { o[0] = fa; o[1] = fb; }
	};
	fused_fft<N, S, 3>(smem, p.tw, -1, ld, st, NoHook{}, threadIdx.x, typename NphiPlan<N>::L{});
}

// ---------------------------------------------------------------------------
// Four-step FFT for nphi = N1 N2 = 96 x 128 = 12288 (theta-contiguous grids).
// With j = j1 + N1 j2 and k = k2 + N2 k1,
//   exp(s 2 pi i j k / N) = w_N^(j1 k2) w_N1^(j1 k1) w_N2^(j2 k2),
// so a length-N transform is N2 transforms of length N1 (over k1), a twiddle
// w_N^(j1 k2), and N1 transforms of length N2 (over k2).  Each CTA runs the
// short transforms of FS_S latitude pairs (one 256-byte run of a grid row per
// element), so its loads and stores are coalesced rows and many CTAs share an
// SM, where the one-pass kernel of this length holds one latitude pair per SM.
// The intermediate lives in grid row j = N1 k2 + j1: the synthesis works in
// place in its output grid (the second step reads and rewrites exactly the
// rows j1 + N1 k2 of its j1), the analysis writes it to a scratch grid.
// The analysis' second step takes k2 and N2 - k2 in one CTA, so that each
// order's pair (z_m, z_{N-m}) is at hand to separate the two real spectra.
constexpr int FS_S = 16;      // latitude pairs per CTA

template <int N1, int N2>
__global__ void __launch_bounds__(Geo<N1, FS_S>::T) fft_fs_synth1_kernel(FftParams p)
{
	extern __shared__ double2 smem[];
	constexpr int N = N1 * N2;
	const int fc = blockIdx.z, k2 = blockIdx.y;
	const int lat0 = blockIdx.x * 2 * FS_S;
	const double2* __restrict__ Ff = p.F + (long)fc * p.fstride;
	const int ml = p.mlim, nlat = p.nlat;
	auto ld = [&](int s, int k1) -> double2 {
		const int ra = lat0 + 2 * s;
		const int j = k2 + N2 * k1;                 // frequency index
		const int k = (j <= ml) ? j : ((j >= N - ml) ? N - j : -1);
		if (k < 0 || ra >= nlat) return make_double2(0.0, 0.0);
		double2 a = __ldg(Ff + (long)k * nlat + ra), b = __ldg(Ff + (long)k * nlat + ra + 1);
		if (k == 0) { a.y = 0.0; b.y = 0.0; }
		return (j <= ml) ? make_double2(a.x - b.y, a.y + b.x) : make_double2(a.x + b.y, b.x - a.y);
	};
	const int c = fc / p.nf;
	double* out = (c == 0 ? p.spat[0] : c == 1 ? p.spat[1] : p.spat[2]) + (long)(fc - c * p.nf) * p.spat_dist;
	auto st = [&](int s, int j1, double2 z) {
		const int row = lat0 + 2 * s;
		if (row >= nlat) return;
		z = cmul(z, __ldg(p.tw + (j1 * k2) % N));
		*reinterpret_cast<double2*>(out + (long)(N1 * k2 + j1) * nlat + row) = z;
	};
	fused_fft<N1, FS_S, 1>(smem, p.tw1, +1, ld, st, NoHook{}, threadIdx.x, typename NphiPlan<N1>::L{});
}

template <int N1, int N2>
__global__ void __launch_bounds__(Geo<N2, FS_S>::T) fft_fs_synth2_kernel(FftParams p)
{
	extern __shared__ double2 smem[];
	const int fc = blockIdx.z, j1 = blockIdx.y;
	const int lat0 = blockIdx.x * 2 * FS_S;
	const int nlat = p.nlat;
	const int c = fc / p.nf;
	double* out = (c == 0 ? p.spat[0] : c == 1 ? p.spat[1] : p.spat[2]) + (long)(fc - c * p.nf) * p.spat_dist;
	auto ld = [&](int s, int k2) -> double2 {
		const int row = lat0 + 2 * s;
		if (row >= nlat) return make_double2(0.0, 0.0);
		return *reinterpret_cast<const double2*>(out + (long)(N1 * k2 + j1) * nlat + row);
	};
	auto st = [&](int s, int j2, double2 z) {
		const int row = lat0 + 2 * s;
		if (row >= nlat) return;
		*reinterpret_cast<double2*>(out + (long)(j1 + N1 * j2) * nlat + row) = z;
	};
	fused_fft<N2, FS_S, 1>(smem, p.tw2, +1, ld, st, NoHook{}, threadIdx.x, typename NphiPlan<N2>::L{});
}

template <int N1, int N2>
__global__ void __launch_bounds__(Geo<N2, FS_S>::T) fft_fs_analys1_kernel(FftParams p)
{
	extern __shared__ double2 smem[];
	constexpr int N = N1 * N2;
	const int fc = blockIdx.z, j1 = blockIdx.y;
	const int lat0 = blockIdx.x * 2 * FS_S;
	const int nlat = p.nlat;
	const int c = fc / p.nf;
	const double* in = (c == 0 ? p.spat_in[0] : c == 1 ? p.spat_in[1] : p.spat_in[2]) + (long)(fc - c * p.nf) * p.spat_dist;
	double* scr = p.scratch + (long)fc * N * nlat;
	auto ld = [&](int s, int j2) -> double2 {
		const int row = lat0 + 2 * s;
		if (row >= nlat) return make_double2(0.0, 0.0);
		return __ldg(reinterpret_cast<const double2*>(in + (long)(j1 + N1 * j2) * nlat + row));
	};
	auto st = [&](int s, int k2, double2 z) {
		const int row = lat0 + 2 * s;
		if (row >= nlat) return;
		double2 w = __ldg(p.tw + (j1 * k2) % N);
		w.y = -w.y;
		*reinterpret_cast<double2*>(scr + (long)(N1 * k2 + j1) * nlat + row) = cmul(z, w);
	};
	fused_fft<N2, FS_S, 1>(smem, p.tw2, -1, ld, st, NoHook{}, threadIdx.x, typename NphiPlan<N2>::L{});
}

template <int N1, int N2>
__global__ void __launch_bounds__(Geo<N1, 2 * FS_S>::T) fft_fs_analys2_kernel(FftParams p)
{
	extern __shared__ double2 smem[];
	using G = Geo<N1, 2 * FS_S>;
	constexpr int N = N1 * N2;
	const int fc = blockIdx.z, ka = blockIdx.y;          // ka = 0 .. N2/2
	const int kb = (N2 - ka) % N2;                        // partner k2 (ka for 0 and N2/2)
	const int lat0 = blockIdx.x * 2 * FS_S;
	const int nlat = p.nlat, ml = p.mlim;
	const double* scr = p.scratch + (long)fc * N * nlat;
	// sequences s < FS_S: k2 = ka, latitude pair s; s >= FS_S: k2 = kb, pair s - FS_S
	auto ld = [&](int s, int j1) -> double2 {
		const int pr = s % FS_S, k2 = (s < FS_S) ? ka : kb;
		const int row = lat0 + 2 * pr;
		if (row >= nlat) return make_double2(0.0, 0.0);
		return *reinterpret_cast<const double2*>(scr + (long)(N1 * k2 + j1) * nlat + row);
	};
	NoHook no;
	fused_fft<N1, 2 * FS_S, 0>(smem, p.tw1, -1, ld, no, NoHook{}, threadIdx.x, typename NphiPlan<N1>::L{});
	// X[at(s, k1)] = z_k, k = k2(s) + N2 k1.  Partner z_{N-k}: for k2 = 0 at
	// (same sequence, (N1 - k1) % N1), else at (other k2, N1 - 1 - k1).
	double2* Ff = p.F + (long)fc * p.fstride;
	const double sc = 0.5 / N;
	const bool self = (ka == kb);
	const int nseq = self ? FS_S : 2 * FS_S;
	for (int e = threadIdx.x; e < nseq * N1; e += G::T) {
		const int s = e / N1, k1 = e - s * N1;
		const int pr = s % FS_S, k2 = (s < FS_S) ? ka : kb;
		const int k = k2 + N2 * k1;
		const int ra = lat0 + 2 * pr;
		if (k > ml || ra >= nlat) continue;
		int sp, kp;
		if (k2 == 0) { sp = s; kp = (N1 - k1) % N1; }
		else { sp = self ? s : (s < FS_S ? s + FS_S : s - FS_S); kp = N1 - 1 - k1; }
		const double2 z = smem[G::at(s, k1)], w = smem[G::at(sp, kp)];
		const double2 fa = make_double2(sc * (z.x + w.x), sc * (z.y - w.y));
		const double2 fb = make_double2(sc * (z.y + w.y), -sc * (z.x - w.x));
		double2* o = Ff + (long)k * nlat + ra;
		asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};"
		             :: "l"(o), "d"(fa.x), "d"(fa.y), "d"(fb.x), "d"(fb.y) : "memory");
	}
}

// ---------------------------------------------------------------------------
// Prefetched fused kernels.  A persistent CTA walks over tiles (2 S latitudes
// of one field-component, tile t = fc * nlg + latitude group) and keeps the
// input of its next tile in flight while the current one is transformed: one
// thread issues tensor copies (TMA, no multicast) of the next tile into a
// shared staging buffer right after the first pass has moved the current
// tile from there into the FFT buffer, and the copies complete on an
// mbarrier that the CTA waits on (bounded) before the next first pass.
//   synthesis input   F[fc][k][theta]: box (2 S latitudes x 2 doubles, <= 256 k)
//   analysis input    theta-contiguous v[f][j][theta]: box (2 S latitudes, 256 or 192 j)
// Outputs are written as by the direct kernels above.
// j rows per box of the analysis input: 256, or nphi for 192, 192 for 384
__host__ __device__ constexpr int box_j(int N) { return (N % 256 == 0) ? 256 : (N <= 256 ? N : 192); }

struct TmaTiles {
	int nlg;          // latitude groups (tiles per field-component)
	int ntiles;
	int ncopy;        // box copies per tile
	int box;          // rows (k or j) per box
	unsigned bytes;   // bytes per tile (all boxes, out-of-range parts included)
	int stage_off;    // staging buffer offset in the dynamic shared memory (bytes)
	int v4;           // F rows 32-byte aligned at even latitudes: one 32-byte store per latitude pair
};

constexpr uint64_t FT_WAIT_NS = 1000000000ull;   // time limit of every mbarrier wait

__device__ int g_fft_wait_err;                    // set when a bounded wait gave up

__device__ __forceinline__ uint32_t su32(const void* ptr) { return static_cast<uint32_t>(__cvta_generic_to_shared(ptr)); }

__device__ __forceinline__ uint64_t gtimer()
{
	uint64_t t;
	asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
	return t;
}

__device__ __forceinline__ bool fbar_wait(uint64_t* bar, uint32_t parity)
{
	const uint32_t a = su32(bar);
	const uint64_t t0 = gtimer();
	for (int it = 0;; it++) {
		if ((it & 1023) == 1023 && gtimer() - t0 > FT_WAIT_NS) return false;
		uint32_t done;
		asm volatile("{\n\t.reg .pred p;\n\t"
		             "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
		             "selp.u32 %0, 1, 0, p;\n\t}"
		             : "=r"(done) : "r"(a), "r"(parity) : "memory");
		if (done) return true;
	}
}

__device__ __forceinline__ void tma_tile3(void* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* bar)
{
	asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
	             :: "r"(su32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(su32(bar))
	             : "memory");
}

// One thread: announce the bytes of a tile, then issue its box copies
// (latitude coordinate c0, rows c * box, field c2).
__device__ __forceinline__ void fetch_tile(uint64_t* bar, const CUtensorMap* map, char* stage, const TmaTiles& tt,
                                           int c0, int c2, int box_bytes)
{
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(su32(bar)), "r"(tt.bytes) : "memory");
	for (int c = 0; c < tt.ncopy; c++)
		tma_tile3(stage + (size_t) c * box_bytes, map, c0, c * tt.box, c2, bar);
}

// Wait for the staged tile; false (uniformly in the CTA) if the wait gave up,
// after recording it and waiting once more (bounded) for the copies in flight.
__device__ __forceinline__ bool stage_ready(uint64_t* bar, uint32_t parity)
{
	const bool ok = fbar_wait(bar, parity);
	if (__syncthreads_or(!ok)) {
		if (threadIdx.x == 0) {
			atomicExch(&g_fft_wait_err, 1);
			fbar_wait(bar, parity);
		}
		return false;
	}
	return true;
}

__device__ __forceinline__ void stage_init(uint64_t* bar)
{
	if (threadIdx.x == 0) {
		asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(su32(bar)) : "memory");
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	__syncthreads();
}

__device__ __forceinline__ void tma_store3(const CUtensorMap* map, const void* src, int c0, int c1, int c2)
{
	asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];"
	             :: "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(su32(src)) : "memory");
}

// tensor stores of this thread have finished reading shared memory
__device__ __forceinline__ void store_reads_done() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }

// Results written to X by every thread become visible to the tensor copies,
// then one thread stores nbox boxes of box_bytes each.
__device__ __forceinline__ void store_tile(const CUtensorMap* map, const char* X, int nbox, int box, int box_bytes, int c0,
                                           int c2)
{
	asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
	__syncthreads();
	if (threadIdx.x == 0) {
		for (int c = 0; c < nbox; c++) tma_store3(map, X + (size_t) c * box_bytes, c0, c * box, c2);
		asm volatile("cp.async.bulk.commit_group;" ::: "memory");
	}
}

// TOUT: theta-contiguous output written by tensor stores of whole tiles
// (rows of 2 S latitudes) from X, instead of 16-byte stores per latitude pair
template <int N, int S, bool TOUT>
__global__ void __launch_bounds__(Geo<N, S>::T, 768 / Geo<N, S>::T) fft4_synth_kernel(
	const __grid_constant__ CUtensorMap fmap, const __grid_constant__ CUtensorMap o0, const __grid_constant__ CUtensorMap o1,
	const __grid_constant__ CUtensorMap o2, FftParams p, TmaTiles tt)
{
	extern __shared__ __align__(128) char fsm[];
	__shared__ __align__(8) uint64_t bar;
	char* base = fsm + ((128u - (su32(fsm) & 127u)) & 127u);   // tensor copies land on 128-byte boundaries
	double2* X = reinterpret_cast<double2*>(base);
	char* stage = base + tt.stage_off;
	const double2* stg = reinterpret_cast<const double2*>(stage);
	const int ml = p.mlim, nlat = p.nlat;
	const int box_bytes = tt.box * 2 * S * 16;
	stage_init(&bar);
	int tile = blockIdx.x;
	if (threadIdx.x == 0) {
		const int fc = tile / tt.nlg;
		fetch_tile(&bar, &fmap, stage, tt, 4 * S * (tile - fc * tt.nlg), fc, box_bytes);
	}
	for (uint32_t parity = 0; tile < tt.ntiles; tile += gridDim.x, parity ^= 1) {
		if (TOUT && threadIdx.x == 0) store_reads_done();     // X is free again (previous tile's stores)
		if (!stage_ready(&bar, parity)) return;
		const int fc = tile / tt.nlg;
		const int lat0 = (tile - fc * tt.nlg) * 2 * S;
		// ml opaque per tile: the first pass's shared addresses and predicates
		// are recomputed per tile instead of held in registers across tiles
		int mlo = ml;
		asm volatile("" : "+r"(mlo));
		auto ld = [&](int s, int j) -> double2 {
			const int k = (j <= mlo) ? j : ((j >= N - mlo) ? N - j : -1);
			if (k < 0) return make_double2(0.0, 0.0);
			// the two latitudes of sequence s, read in an order that alternates
			// with the row so that the 8 lanes of a shared-memory phase (4 rows)
			// hit distinct banks; swapped back in registers
			const int f = (k >> (S == 1 ? 2 : (S == 2 ? 1 : 0))) & 1;
			const double2 u0 = stg[k * 2 * S + 2 * s + f], u1 = stg[k * 2 * S + 2 * s + 1 - f];
			double2 a = f ? u1 : u0, b = f ? u0 : u1;
			if (k == 0) { a.y = 0.0; b.y = 0.0; }
			return (j <= mlo) ? make_double2(a.x - b.y, a.y + b.x) : make_double2(a.x + b.y, b.x - a.y);
		};
		const int c = fc / p.nf;
		const int next = tile + gridDim.x;
		auto prefetch = [&]() {
			if (threadIdx.x == 0 && next < tt.ntiles) {
				asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
				const int nfc = next / tt.nlg;
				fetch_tile(&bar, &fmap, stage, tt, 4 * S * (next - nfc * tt.nlg), nfc, box_bytes);
			}
		};
		if constexpr (TOUT) {
			int dummy = 0;
			auto st = [&](int, int, double2) { dummy++; };
			fused_fft<N, S, 2>(X, p.tw, +1, ld, st, prefetch, threadIdx.x, typename NphiPlan<N>::L{});
			constexpr int BJ = box_j(N);
			const CUtensorMap* om = (c == 0) ? &o0 : (c == 1 ? &o1 : &o2);
			store_tile(om, base, N / BJ, BJ, BJ * S * 16, lat0, fc - c * p.nf);
		} else {
			double* out = (c == 0 ? p.spat[0] : c == 1 ? p.spat[1] : p.spat[2]) + (long)(fc - c * p.nf) * p.spat_dist;
			const bool phi = p.phi_contiguous, v2 = p.vec2;
			auto st = [&](int s, int j, double2 z) {
				const int row = lat0 + 2 * s;
				if (row >= nlat) return;
				if (!phi) {
					double* o = out + (long)j * nlat + row;
					if (v2) *reinterpret_cast<double2*>(o) = z;
					else { o[0] = z.x; o[1] = z.y; }
				} else {
					out[(long)row * N + j] = z.x;
					out[(long)(row + 1) * N + j] = z.y;
				}
			};
			fused_fft<N, S, 1>(X, p.tw, +1, ld, st, prefetch, threadIdx.x, typename NphiPlan<N>::L{});
		}
	}
	if (TOUT && threadIdx.x == 0) store_reads_done();
}

template <int N, int S>
__global__ void __launch_bounds__(Geo<N, S>::T, 768 / Geo<N, S>::T) fft4_analys_kernel(
	const __grid_constant__ CUtensorMap m0, const __grid_constant__ CUtensorMap m1, const __grid_constant__ CUtensorMap m2,
	FftParams p, TmaTiles tt)
{
	using G = Geo<N, S>;
	extern __shared__ __align__(128) char fsm[];
	__shared__ __align__(8) uint64_t bar;
	char* base = fsm + ((128u - (su32(fsm) & 127u)) & 127u);   // tensor copies land on 128-byte boundaries
	double2* X = reinterpret_cast<double2*>(base);
	char* stage = base + tt.stage_off;
	const double* stg = reinterpret_cast<const double*>(stage);
	const int nlat = p.nlat, nf = p.nf;
	const int box_bytes = box_j(N) * 2 * S * 8;
	auto issue = [&](int t) {
		const int fc = t / tt.nlg, c = fc / nf;
		const CUtensorMap* m = (c == 0) ? &m0 : (c == 1 ? &m1 : &m2);
		fetch_tile(&bar, m, stage, tt, 2 * S * (t - fc * tt.nlg), fc - c * nf, box_bytes);
	};
	stage_init(&bar);
	int tile = blockIdx.x;
	if (threadIdx.x == 0) issue(tile);
	for (uint32_t parity = 0; tile < tt.ntiles; tile += gridDim.x, parity ^= 1) {
		if (!stage_ready(&bar, parity)) return;
		const int fc = tile / tt.nlg;
		const int lat0 = (tile - fc * tt.nlg) * 2 * S;
		int rs = 2 * S;                         // opaque per tile, as mlim in the synthesis
		asm volatile("" : "+r"(rs));
		auto ld = [&](int s, int j) -> double2 { return *reinterpret_cast<const double2*>(stg + j * rs + 2 * s); };
		const int next = tile + gridDim.x;
		auto prefetch = [&]() {
			if (threadIdx.x == 0 && next < tt.ntiles) {
				asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
				issue(next);
			}
		};
		// Fourier rows straight from the last radix pass: F_k of the two
		// latitudes of sequence s from (z_k, z_{N-k}), one 32-byte store
		double2* Ff = p.F + (long)fc * p.fstride;
		const double sc = 0.5 / N;
		const int ml = p.mlim;
		auto st = [&](int s, int k, double2 z, double2 w) {
			const int ra = lat0 + 2 * s;
			if (k > ml || ra >= nlat) return;
			const double2 fa = make_double2(sc * (z.x + w.x), sc * (z.y - w.y));
			const double2 fb = make_double2(sc * (z.y + w.y), -sc * (z.x - w.x));
			double2* o = Ff + (long)k * nlat + ra;
			if (tt.v4)
				asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};"
				             :: "l"(o), "d"(fa.x), "d"(fa.y), "d"(fb.x), "d"(fb.y) : "memory");
			else { o[0] = fa; o[1] = fb; }
		};
		fused_fft<N, S, 3>(X, p.tw, -1, ld, st, prefetch, threadIdx.x, typename NphiPlan<N>::L{});
	}
}

// the driver's tensor-map encoder, resolved once (thread-safe static initialisation)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
	static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
		void* f = nullptr;
		cudaDriverEntryPointQueryResult q;
		if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
		    q == cudaDriverEntryPointSuccess)
			return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
		cudaGetLastError();
		return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
	}();
	return fn;
}

// 3-d FP64 tensor map, dims / byte strides of dims 1 and 2 / box, no swizzle,
// zero fill out of range
bool encode3(CUtensorMap* m, const void* base, uint64_t d0, uint64_t d1, uint64_t d2, uint64_t s1, uint64_t s2,
             uint32_t b0, uint32_t b1)
{
	PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
	if (!enc || ((uintptr_t) base & 15) || (s1 & 15) || (s2 & 15) || ((b0 * 8) & 15)) return false;
	const cuuint64_t dims[3] = {d0, d1, d2};
	const cuuint64_t strides[2] = {s1, s2};
	const cuuint32_t box[3] = {b0, b1, 1};
	const cuuint32_t es[3] = {1, 1, 1};
	return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void*>(base), dims, strides, box, es,
	           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
	           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int sm_count()
{
	static const int n = [] {
		int dev = 0, c = 0;
		cudaGetDevice(&dev);
		if (cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || c <= 0) { cudaGetLastError(); c = 148; }
		return c;
	}();
	return n;
}

// F[fc][k][theta] as FP64 rows of 2 nlat doubles: box (2 S latitudes, box k)
bool f_map(CUtensorMap* m, const FftParams& p, int nfc, int S, int box)
{
	return encode3(m, p.F, 2 * (uint64_t) p.nlat, p.mlim + 1, nfc, 16 * (uint64_t) p.nlat, 16 * (uint64_t) p.fstride, 4 * S, box);
}

// theta-contiguous spatial component c: dims (nlat, nphi, fields)
bool grid_map(CUtensorMap* m, const double* base, const FftParams& p, int N, int S)
{
	return encode3(m, base, p.nlat, N, p.nf, 8 * (uint64_t) p.nlat, 8 * (uint64_t) p.spat_dist, 2 * S, box_j(N));
}

template <int N, int S>
bool launch_fft4(const FftParams& p, int nfc, cudaStream_t st, bool synth)
{
	using G = Geo<N, S>;
	alignas(64) CUtensorMap maps[4];        // synthesis: F, output components; analysis: input components
	TmaTiles tt;
	tt.nlg = (p.nlat + 2 * S - 1) / (2 * S);
	tt.ntiles = tt.nlg * nfc;
	const int rows = p.mlim + 1;
	const int kbox = rows < 256 ? rows : 256;            // k rows per box of F
	const int ncomp = (nfc + p.nf - 1) / p.nf;
	// tensor maps over the theta-contiguous grid (16-byte aligned, even nlat)
	const bool grid_ok = p.vec2 && !p.phi_contiguous && !(p.nlat & 1) && N % box_j(N) == 0;
	const bool tstore = (p.generic != 3);               // option 3 = 3: prefetched loads, direct stores
	bool tout = false;
	size_t stage_bytes;
	if (synth) {
		tt.box = kbox;
		tt.ncopy = (rows + tt.box - 1) / tt.box;
		stage_bytes = (size_t) tt.ncopy * tt.box * 2 * S * 16;
		if (!f_map(&maps[0], p, nfc, S, tt.box)) return false;
		tout = grid_ok && tstore;
		for (int c = 0; c < 3 && tout; c++) tout = grid_map(&maps[1 + c], p.spat[c < ncomp ? c : 0], p, N, S);
	} else {
		// theta-contiguous grids only (phi-contiguous rows are read faster
		// straight from global memory by the direct kernel)
		if (!grid_ok) return false;
		tt.box = box_j(N);
		tt.ncopy = N / tt.box;
		stage_bytes = (size_t) N * 2 * S * 8;
		for (int c = 0; c < 3; c++)
			if (!grid_map(&maps[c], p.spat_in[c < ncomp ? c : 0], p, N, S)) return false;
	}
	tt.bytes = (unsigned) (stage_bytes + p.extra_tx);
	tt.v4 = !((uintptr_t) p.F & 31) && !(p.nlat & 1) && !(p.fstride & 1);
	tt.stage_off = (int)(((size_t) S * G::SEQ * sizeof(double2) + 127) / 128 * 128);
	const size_t smem = tt.stage_off + stage_bytes + 128;
	if (smem > 226 * 1024) return false;
	const void* fn = synth ? (tout ? (const void*) fft4_synth_kernel<N, S, true> : (const void*) fft4_synth_kernel<N, S, false>)
	                       : (const void*) fft4_analys_kernel<N, S>;
	int per_sm = 0;
	if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, G::T, smem) != cudaSuccess || per_sm <= 0) {
		cudaGetLastError();
		return false;
	}
	const int grid = std::min(tt.ntiles, per_sm * sm_count());
	if (synth) {
		if (tout) fft4_synth_kernel<N, S, true><<<grid, G::T, smem, st>>>(maps[0], maps[1], maps[2], maps[3], p, tt);
		else fft4_synth_kernel<N, S, false><<<grid, G::T, smem, st>>>(maps[0], maps[0], maps[0], maps[0], p, tt);
	} else {
		fft4_analys_kernel<N, S><<<grid, G::T, smem, st>>>(maps[0], maps[1], maps[2], p, tt);
	}
	return true;
}

template <int N, int S>
bool launch_fft3(const FftParams& p, int nfc, cudaStream_t st, bool synth)
{
	using G = Geo<N, S>;
	const size_t smem = sizeof(double2) * (size_t) S * G::SEQ;
	dim3 grid((p.nlat + 2 * S - 1) / (2 * S), nfc);
	if (synth) fft3_synth_kernel<N, S><<<grid, G::T, smem, st>>>(p);
	else fft3_analys_kernel<N, S><<<grid, G::T, smem, st>>>(p);
	return true;
}

template <int N>
bool launch_fft3_n(const FftParams& p, int nfc, cudaStream_t st, bool synth)
{
	// latitude pairs per CTA: 8 (full 128-byte lines of a theta-contiguous
	// grid, two butterflies per thread) where the buffer fits, else up to 4
	// while the block stays at <= 768 threads
	if constexpr (8 * (N + (N >> 3) + 1) * 16 <= 227 * 1024) if (p.S >= 8) return launch_fft3<N, 8>(p, nfc, st, synth);
	if constexpr (4 * N / 8 <= 768) if (p.S >= 4) return launch_fft3<N, 4>(p, nfc, st, synth);
	if constexpr (2 * N / 8 <= 768) if (p.S >= 2) return launch_fft3<N, 2>(p, nfc, st, synth);
	return launch_fft3<N, 1>(p, nfc, st, synth);
}

} // namespace

// kernel family of the last FFT launch in the process (a diagnostic, any
// thread), and whether the launch in progress on this thread took the
// prefetching kernels
static std::atomic<int> g_last_fft_path{-1};
static thread_local bool g_fft4_ran = false;

namespace {

// prefetched kernels for the automatic choice (p.generic == 0); false where
// they do not apply (layout, alignment, shared memory), for the direct ones
template <int N>
bool launch_fft4_n(const FftParams& p, int nfc, cudaStream_t st, bool synth)
{
	if constexpr (N + (N >> 3) + 8 > 6400) return false;     // FFT buffer above 100 KB
	else {
		if (p.S == 1) return launch_fft4<N, 1>(p, nfc, st, synth);
		if constexpr (2 * N / 8 <= 768) if (p.S == 2) return launch_fft4<N, 2>(p, nfc, st, synth);
		if constexpr (4 * N / 8 <= 768) if (p.S == 4) return launch_fft4<N, 4>(p, nfc, st, synth);
		return false;
	}
}

// four-step path: nphi = 12288 on theta-contiguous grids with 16-byte
// aligned latitude pairs and (analysis) a scratch grid; false otherwise
bool launch_fourstep(const FftParams& p, int nfc, cudaStream_t st, bool synth)
{
	constexpr int N1 = 96, N2 = 128;
	if (p.N != N1 * N2 || p.phi_contiguous || !p.vec2 || !p.tw1 || p.generic != 0 || (!synth && !p.scratch)) return false;
	if (p.nlat % 2 || ((uintptr_t) p.F & 31)) return false;
	using G1 = Geo<N1, FS_S>;
	using G2 = Geo<N2, FS_S>;
	using G3 = Geo<N1, 2 * FS_S>;
	const size_t s1 = sizeof(double2) * (size_t) FS_S * G1::SEQ, s2 = sizeof(double2) * (size_t) FS_S * G2::SEQ;
	const size_t s3 = sizeof(double2) * (size_t)(2 * FS_S) * G3::SEQ;
	static bool attr = false;
	if (!attr) {
		cudaFuncSetAttribute(fft_fs_analys2_kernel<N1, N2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) s3);
		attr = true;
	}
	const int nlb = (p.nlat + 2 * FS_S - 1) / (2 * FS_S);
	if (synth) {
		fft_fs_synth1_kernel<N1, N2><<<dim3(nlb, N2, nfc), G1::T, s1, st>>>(p);
		fft_fs_synth2_kernel<N1, N2><<<dim3(nlb, N1, nfc), G2::T, s2, st>>>(p);
	} else {
		fft_fs_analys1_kernel<N1, N2><<<dim3(nlb, N1, nfc), G2::T, s2, st>>>(p);
		fft_fs_analys2_kernel<N1, N2><<<dim3(nlb, N2 / 2 + 1, nfc), G3::T, s3, st>>>(p);
	}
	shtb_count_launch();         // the second of the two launches is counted by the caller
	return true;
}

bool launch_fused(const FftParams& p, int nfc, cudaStream_t st, bool synth)
{
	if (launch_fourstep(p, nfc, st, synth)) return true;
	if (p.generic == 0 || p.generic == 3) {
		bool done = false;
		switch (p.N) {
			case 192: done = launch_fft4_n<192>(p, nfc, st, synth); break;
			case 384: done = launch_fft4_n<384>(p, nfc, st, synth); break;
			case 768: done = launch_fft4_n<768>(p, nfc, st, synth); break;
			case 1536: done = launch_fft4_n<1536>(p, nfc, st, synth); break;
			case 3072: done = launch_fft4_n<3072>(p, nfc, st, synth); break;
			case 6144: done = launch_fft4_n<6144>(p, nfc, st, synth); break;
			default: break;
		}
		if (done) { g_fft4_ran = true; return true; }
	}
	switch (p.N) {
		case 192: return launch_fft3_n<192>(p, nfc, st, synth);
		case 384: return launch_fft3_n<384>(p, nfc, st, synth);
		case 768: return launch_fft3_n<768>(p, nfc, st, synth);
		case 1536: return launch_fft3_n<1536>(p, nfc, st, synth);
		case 3072: return launch_fft3_n<3072>(p, nfc, st, synth);
		case 6144: return launch_fft3_n<6144>(p, nfc, st, synth);
		case 12288: return launch_fft3_n<12288>(p, nfc, st, synth);
		default: return false;
	}
}

template <int N, int S>
void set_fft4_limits(int lim)
{
	cudaFuncSetAttribute(fft4_synth_kernel<N, S, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
	cudaFuncSetAttribute(fft4_synth_kernel<N, S, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
	cudaFuncSetAttribute(fft4_analys_kernel<N, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
}

template <int N>
void set_fused_limits()
{
	const int lim = 227 * 1024;
	if constexpr (N + (N >> 3) + 8 <= 6400) {
		// the prefetching kernels also hold an mbarrier in static shared memory
		const int lim4 = 226 * 1024;
		set_fft4_limits<N, 1>(lim4);
		if constexpr (2 * N / 8 <= 768) set_fft4_limits<N, 2>(lim4);
		if constexpr (4 * N / 8 <= 768) set_fft4_limits<N, 4>(lim4);
	}
	cudaFuncSetAttribute(fft3_synth_kernel<N, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
	cudaFuncSetAttribute(fft3_analys_kernel<N, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
	if constexpr (2 * N / 8 <= 768) {
		cudaFuncSetAttribute(fft3_synth_kernel<N, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
		cudaFuncSetAttribute(fft3_analys_kernel<N, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
	}
	if constexpr (4 * N / 8 <= 768) {
		cudaFuncSetAttribute(fft3_synth_kernel<N, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
		cudaFuncSetAttribute(fft3_analys_kernel<N, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
	}
	if constexpr (8 * (N + (N >> 3) + 1) * 16 <= 227 * 1024) {
		cudaFuncSetAttribute(fft3_synth_kernel<N, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
		cudaFuncSetAttribute(fft3_analys_kernel<N, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
	}
}

} // namespace

static int seq_len_host(int N, int S)
{
	const int a = N + (N >> 3);
	return a + (((S >= 8 ? 1 : 8 / S) - a) & 7);
}

int fft_threads(int N, int S, unsigned long long rcode, int nradix)
{
	(void) rcode; (void) nradix;
	// about one radix-8 butterfly per thread
	int T = (S * N / 8 + 31) / 32 * 32;
	return T < 64 ? 64 : (T > 768 ? 768 : T);
}

size_t fft_smem_bytes(int N, int S) { return 2 * sizeof(double2) * (size_t) S * seq_len_host(N, S); }

// sizes with a fused pass chain (one in-place buffer: these may exceed the
// generic kernels' two-buffer limit)
bool fft_fused_available(int N)
{
	switch (N) {
		case 192: case 384: case 768: case 1536: case 3072: case 6144: case 12288: return true;
		default: return false;
	}
}

// kernel family of the last FFT launch (host side): 0 generic, 1 fused
// direct loads, 2 fused with prefetched tiles
int fft_last_path() { return g_last_fft_path.load(); }

void launch_fft_synth(const FftParams& p, int nfc, cudaStream_t st)
{
	g_fft4_ran = false;
	if (p.generic != 1 && launch_fused(p, nfc, st, true)) { g_last_fft_path = g_fft4_ran ? 2 : 1; shtb_count_launch(); return; }
	g_last_fft_path = 0;
	const int T = fft_threads(p.N, p.S, p.rcode, p.nradix);
	const size_t smem = fft_smem_bytes(p.N, p.S);
	dim3 grid((p.nlat + 2 * p.S - 1) / (2 * p.S), nfc);
	switch (p.S) {
		case 4: fft_synth_kernel<4><<<grid, T, smem, st>>>(p); break;
		case 2: fft_synth_kernel<2><<<grid, T, smem, st>>>(p); break;
		default: fft_synth_kernel<1><<<grid, T, smem, st>>>(p); break;
	}
	shtb_count_launch();
}

void launch_fft_analys(const FftParams& p, int nfc, cudaStream_t st)
{
	g_fft4_ran = false;
	if (p.generic != 1 && launch_fused(p, nfc, st, false)) { g_last_fft_path = g_fft4_ran ? 2 : 1; shtb_count_launch(); return; }
	g_last_fft_path = 0;
	const int T = fft_threads(p.N, p.S, p.rcode, p.nradix);
	const size_t smem = fft_smem_bytes(p.N, p.S);
	dim3 grid((p.nlat + 2 * p.S - 1) / (2 * p.S), nfc);
	switch (p.S) {
		case 4: fft_analys_kernel<4><<<grid, T, smem, st>>>(p); break;
		case 2: fft_analys_kernel<2><<<grid, T, smem, st>>>(p); break;
		default: fft_analys_kernel<1><<<grid, T, smem, st>>>(p); break;
	}
	shtb_count_launch();
}

void fft_set_smem_limits()
{
	tensor_map_encoder();    // resolved here, outside any stream capture
	sm_count();
	set_fused_limits<192>(); set_fused_limits<384>(); set_fused_limits<768>();
	set_fused_limits<1536>(); set_fused_limits<3072>(); set_fused_limits<6144>(); set_fused_limits<12288>();
	const int lim = 227 * 1024;
	cudaFuncSetAttribute(fft_synth_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
	cudaFuncSetAttribute(fft_synth_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
	cudaFuncSetAttribute(fft_synth_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
	cudaFuncSetAttribute(fft_analys_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
	cudaFuncSetAttribute(fft_analys_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
	cudaFuncSetAttribute(fft_analys_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
}

// Returns (and clears) the flag that a bounded wait of the prefetched FFT
// kernels gave up; waits for the device.
int fft_take_wait_error()
{
	int e = 0;
	cudaDeviceSynchronize();
	if (cudaMemcpyFromSymbol(&e, g_fft_wait_err, sizeof(int)) != cudaSuccess) { cudaGetLastError(); return 0; }
	if (e) {
		const int z = 0;
		cudaMemcpyToSymbol(g_fft_wait_err, &z, sizeof(int));
	}
	return e;
}
