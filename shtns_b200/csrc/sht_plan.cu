// Plan creation and destruction for shtns_b200 (host C++ with CUDA runtime).
//
// Mirrors the reference's shtns_create / shtns_set_grid (sht_init.c:1085-1500):
// sizes and index arrays, Legendre recurrence tables (sht_legendre.c:558-736),
// Gauss grid (sht_legendre.c:763-811, sht_init.c:560-649), polar threshold
// (sht_init.c:522-557) and the vector coupling matrices (sht_func.c:400-447).
// The tables go to the GPU once per plan, where the recurrence checkpoints are
// generated in FP64.
#include "sht_internal.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <atomic>

// ---------------------------------------------------------------------------
// error state
static int g_return_errors = 0;
static thread_local std::string g_last_error;
static thread_local int g_status = 0;
static int g_verbose = 0;
static std::atomic<long> g_launches{0};

void shtb_set_error(int code, const std::string& msg)
{
	g_last_error = msg;
	if (g_status == 0) g_status = code;
	if (g_verbose) fprintf(stderr, "[shtns_b200] %s\n", msg.c_str());
}

void shtb_count_launch(int n) { g_launches += n; }

bool shtb_cuda_ok(cudaError_t e, const char* where)
{
	if (e == cudaSuccess) return true;
	shtb_set_error(2, std::string(where) + ": " + cudaGetErrorString(e));
	return false;
}

// Plan-level failure: like shtns_runerr (sht_init.c:67-72) unless the caller
// asked for error returns.
static void plan_error(const std::string& msg)
{
	g_last_error = msg;
	if (!g_return_errors) {
		fprintf(stderr, "\n *** [SHTns-B200] Run-time error : %s\n", msg.c_str());
		exit(1);
	}
	if (g_verbose) fprintf(stderr, "[shtns_b200] %s\n", msg.c_str());
}

extern "C" void shtns_b200_error_mode(int return_errors) { g_return_errors = return_errors; }
extern "C" const char* shtns_b200_last_error(void) { return g_last_error.c_str(); }
extern "C" int shtns_b200_status(void) { int s = g_status; g_status = 0; return s; }
extern "C" long shtns_b200_launch_count(void) { return g_launches.load(); }
extern "C" void shtns_verbose(int v) { g_verbose = v; }
extern "C" void shtns_print_version(void) { printf("[SHTns-B200] spherical harmonic transforms for sm_100a, SHTns 3.5.2 API\n"); }
extern "C" const char* shtns_get_build_info(void) { return "[SHTns-B200] sm_100a, FP64 tensor-core Legendre, SHTns 3.5.2 API"; }

extern "C" long nlm_calc(long lmax, long mmax, long mres)
{
	if (mmax * mres > lmax) mmax = lmax / mres;
	return (mmax + 1) * (lmax + 1) - mres * (mmax * (mmax + 1)) / 2;
}

extern "C" long nlm_cplx_calc(long lmax, long mmax, long mres)
{
	if (mres != 1) return 0;
	if (mmax > lmax) mmax = lmax;
	return (lmax + 1) * (lmax + 1) - (lmax - mmax) * (lmax - mmax + 1);
}

// ---------------------------------------------------------------------------
// chained list of live plans (shtns_reset destroys them all)
static std::mutex g_plans_mu;
static std::vector<shtns_cfg> g_plans;
static int g_gpu_id = 0;

extern "C" int shtns_use_threads(int num_threads) { (void) num_threads; return 1; }

extern "C" int shtns_use_gpu(int device_id)
{
	int count = 0;
	if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return -1;
	if (device_id < 0) return -1;
	g_gpu_id = device_id % count;
	cudaSetDevice(g_gpu_id);
	return g_gpu_id;
}

// ---------------------------------------------------------------------------
// Legendre tables of the classic recurrence in the degree at fixed order m,
//   P_l = a_l x P_{l-1} + b_l P_{l-2},   P_{m+1} = a_{m+1} x P_m,
//   P_m = c_m sin^m(theta),
// for the two normalisations of the API (standard results, e.g. Abramowitz &
// Stegun 8.5.3 rescaled):
//   orthonormal:  a_l = sqrt((4 l^2 - 1) / (l^2 - m^2)),
//                 b_l = -sqrt((2 l + 1) ((l-1)^2 - m^2) / ((2 l - 3) (l^2 - m^2))),
//                 c_m = sqrt(prod_{j=1..m} (2 j + 1) / (2 j) / (4 pi));
//   Schmidt:      a_l = (2 l - 1) / sqrt(l^2 - m^2),
//                 b_l = -sqrt(((l-1)^2 - m^2) / (l^2 - m^2)),
//                 c_m = sqrt(prod_{j=1..m} (2 j + 1) / (2 j) / (2 m + 1));
//   4 pi-normalised: the orthonormal a_l, b_l and c_m times sqrt(4 pi),
// times the order renormalisation for m > 0 and the Condon-Shortley sign
// (-1)^m when asked for.  Storage per order (the pair layout the local
// evaluation kernels read): pair 0 = (c_m, a_{m+1}), pair j >= 1 =
// (b_{m+j+1}, a_{m+j+1}), up to degree lmax + 1; all in long double.
static void legendre_tables(shtns_cfg s)
{
	const int lmax = s->lmax, mmax = s->mmax, mres = s->mres;
	const bool schmidt = (s->base_norm == sht_schmidt);
	s->alm_off.resize(mmax + 2);
	long tot = 0;
	for (int im = 0; im <= mmax; im++) { s->alm_off[im] = tot; tot += 2 * (lmax + 2 - im * mres); }
	s->alm_off[mmax + 1] = tot;
	s->alm.assign(tot + 2, 0.0);
	const long double four_pi = 4.0L * 3.14159265358979323846264338327950288L;
	long double prod = 1.0L;              // prod_{j=1..m} (2j+1)/(2j), advanced with m
	int mprod = 0;
	for (int im = 0; im <= mmax; im++) {
		const long m = (long) im * mres;
		while (mprod < m) { mprod++; prod *= ((long double) mprod + 0.5L) / (long double) mprod; }
		long double c2 = prod * ((s->base_norm == sht_orthonormal) ? 1.0L / four_pi : 1.0L);
		if (m > 0) c2 *= (long double) s->mpos_renorm;
		long double c = std::sqrt(c2);
		if (schmidt) c /= std::sqrt((long double)(2 * m + 1));
		if ((m & 1) && s->cs_phase) c = -c;
		const auto a_l = [&](long l) -> long double {
			const long double d = (long double)((l - m) * (l + m));
			return schmidt ? (2 * l - 1) / std::sqrt(d) : std::sqrt((long double)((2 * l + 1) * (2 * l - 1)) / d);
		};
		const auto b_l = [&](long l) -> long double {
			const long double d = (long double)((l - m) * (l + m)), d1 = (long double)((l - 1 - m) * (l - 1 + m));
			return schmidt ? -std::sqrt(d1) / std::sqrt(d)
			               : -std::sqrt(((2 * l + 1) * d1) / ((long double)(2 * l - 3) * d));
		};
		double* al = s->alm.data() + s->alm_off[im];
		al[0] = (double) c;
		al[1] = (double) a_l(m + 1);
		for (long l = m + 2, j = 2; l <= lmax + 1; l++, j += 2) {
			al[j] = (double) b_l(l);
			al[j + 1] = (double) a_l(l);
		}
	}
}

// a_l of order im for degree l (m < l <= lmax+1)
static inline double alm_a(shtns_cfg s, int im, int l)
{
	const int m = im * s->mres;
	return s->alm[s->alm_off[im] + 2 * (l - m - 1) + 1];
}
static inline double alm_b(shtns_cfg s, int im, int l)   // l >= m+2
{
	const int m = im * s->mres;
	return s->alm[s->alm_off[im] + 2 * (l - m - 1)];
}

// Coefficients of cos(theta) x Q coupling degrees l-1 and l+1 (mul_ct_matrix,
// sht_func.c:395-458): mx[2 lm] multiplies Q_{l-1}, mx[2 lm + 1] Q_{l+1};
// zero for l = m (below) and l = lmax (above).  st_dt_matrix scales them by
// (l - 1) and -(l + 2) for sin(theta) d/dtheta (sht_func.c:460-469).
static void ct_coefficients(shtns_cfg s, double* mx, int stdt)
{
	long lm = 0;
	for (int im = 0; im <= s->mmax; im++) {
		const int m = im * s->mres;
		for (int l = m; l <= s->lmax; l++, lm++) {
			double lo = (l > m) ? 1.0 / alm_a(s, im, l) : 0.0, hi = 0.0;
			if (l < s->lmax)
				hi = (s->base_norm == sht_schmidt) ? -alm_b(s, im, l + 2) / alm_a(s, im, l + 2) : 1.0 / alm_a(s, im, l + 1);
			if (stdt) { lo *= (l - 1); hi *= -(l + 2); }
			mx[2 * lm] = lo;
			mx[2 * lm + 1] = hi;
		}
	}
}

extern "C" void mul_ct_matrix(shtns_cfg s, double* mx) { if (s && mx) ct_coefficients(s, mx, 0); }
extern "C" void st_dt_matrix(shtns_cfg s, double* mx) { if (s && mx) ct_coefficients(s, mx, 1); }

// Ishioka's recurrence (J. Meteor. Soc. Japan 96, 241-249, 2018,
// doi:10.2151/jmsj.2018-019), derived here for the orthonormal functions.
// With eps_l = sqrt((l^2 - m^2) / (4 l^2 - 1)), x P_l = eps_{l+1} P_{l+1} +
// eps_l P_{l-1}.  Writing the odd degrees as P_{m+2k+1} = x p0 d_k Y_k (p0 the
// seed c_m, Y_0 = sin^m(theta)) and applying the three-term relation twice
// gives a two-term recurrence in x^2 for Y_k; choosing
//   d_0 = 1 / eps_{m+1},   d_{k+1} = (-1)^k / (d_k eps_{m+2k+2} eps_{m+2k+3})
// makes the coefficient of Y_{k-1} equal to one:
//   Y_{k+1} = (C_{2k+1} x^2 + C_{2k}) Y_k + Y_{k-1},
//   C_{2k+1} = (-1)^k d_k^2,   C_{2k} = -C_{2k+1} (eps_{m+2k+1}^2 + eps_{m+2k+2}^2).
// The even degrees follow from x P_{m+2k} = eps_{m+2k+1} P_{m+2k+1} +
// eps_{m+2k} P_{m+2k-1}:
//   P_{m+2k} = p0 (eps_{m+2k+1} d_k Y_k + eps_{m+2k} d_{k-1} Y_{k-1}),
// so a field sum_l Q_l P_l = sum_k (X0_k Q_{m+2k} + X1_k Q_{m+2k+2}) Y_k +
// x sum_k X2_k Q_{m+2k+1} Y_k with
//   X0_k = p0 eps_{m+2k+1} d_k,  X1_k = p0 eps_{m+2k+2} d_k,  X2_k = p0 d_k.
// Schmidt functions are the orthonormal ones times sqrt(4 pi / (2l + 1)) up to
// the seed: the same Y_k, with the synthesis coefficient of degree l divided
// by sqrt(2 l + 1) (and p0 the orthonormal seed) and the analysis one
// multiplied by it.  Per order: C (2 per k, padded so that kernels may read
// whole 32-step segments) and the basis change X (3 per k) for synthesis (xs)
// and analysis (xa).  (The reference builds the same recurrence in
// sht_legendre.c:673-734.)
static void ishioka_tables(shtns_cfg s)
{
	const int lmax = s->lmax, mmax = s->mmax, mres = s->mres;
	s->kmax_h.resize(mmax + 1);
	s->koff_h.resize(mmax + 1); s->coff_h.resize(mmax + 1); s->xoff_h.resize(mmax + 1);
	s->voff_h.resize(mmax + 1); s->ckoff_h.resize(mmax + 1);
	long kt = 0, ct = 0, xt = 0, vt = 0;
	for (int im = 0; im <= mmax; im++) {
		const int m = im * mres;
		const int kmax = (lmax + 1 - m) / 2 + 1;         // Y_k rows for degrees up to lmax+1
		const int nseg = (kmax + LG_SEG - 1) / LG_SEG;     // coefficient padding: whole 32-step chunks
		s->kmax_h[im] = kmax;
		s->koff_h[im] = (int) kt;  kt += kmax;
		s->coff_h[im] = (int) ct;  ct += 2 * (nseg * LG_SEG + 2);
		s->xoff_h[im] = (int) xt;  xt += 3 * (kmax + 1);
		s->voff_h[im] = (int) vt;  vt += lmax + 3 - m;
	}
	s->ktot = kt; s->ctot = ct; s->xtot = xt; s->vtot = vt; s->segtot = 0;
	s->ish_c.assign(ct, 0.0);
	s->ish_xs.assign(xt, 0.0);
	s->ish_xa.assign(xt, 0.0);
	const bool schmidt = (s->base_norm == sht_schmidt);
	for (int im = 0; im <= mmax; im++) {
		const long m = (long) im * mres;
		const auto eps = [&](long l) -> long double {
			return std::sqrt((long double)((l - m) * (l + m)) / (long double)((2 * l + 1) * (2 * l - 1)));
		};
		// degree-l scale of the Schmidt basis change (1 for orthonormal functions)
		const auto nrm = [&](long l) -> long double { return schmidt ? std::sqrt((long double)(2 * l + 1)) : 1.0L; };
		long double p0 = s->alm[s->alm_off[im]];
		if (schmidt) p0 *= std::sqrt((long double)(2 * m + 1));     // the orthonormal seed
		const long nk = (lmax - m + 1) / 2;                            // C for k < nk, X for k <= nk
		double* c = s->ish_c.data() + s->coff_h[im];
		double* xs = s->ish_xs.data() + s->xoff_h[im];
		double* xa = s->ish_xa.data() + s->xoff_h[im];
		long double d = 1.0L / eps(m + 1);
		for (long k = 0; k <= nk; k++) {
			const long l = m + 2 * k;
			const long double x0 = p0 * eps(l + 1) * d, x1 = p0 * eps(l + 2) * d, x2 = p0 * d;
			xs[3 * k] = (double)(x0 / nrm(l));     xa[3 * k] = (double)(x0 * nrm(l));
			xs[3 * k + 1] = (double)(x1 / nrm(l + 2)); xa[3 * k + 1] = (double)(x1 * nrm(l + 2));
			xs[3 * k + 2] = (double)(x2 / nrm(l + 1)); xa[3 * k + 2] = (double)(x2 * nrm(l + 1));
			if (k < nk) {
				const long double sgn = (k & 1) ? -1.0L : 1.0L;
				const long double c1 = sgn * d * d;
				const long double e1 = eps(l + 1), e2 = eps(l + 2);
				c[2 * k + 1] = (double) c1;
				c[2 * k] = (double)(-c1 * (e1 * e1 + e2 * e2));
			}
			d = ((k & 1) ? -1.0L : 1.0L) / (d * eps(l + 2) * eps(l + 3));
		}
	}
}

// Coupling coefficients of cos(theta), sin(theta) d/dtheta and
// 2 cos + sin d/dtheta, per degree l = m..lmax+1 (sht_func.c:400-447,
// sht_init.c:1378-1387): lo = coefficient of X_{l-1}, hi = of X_{l+1}.
static void vector_tables(shtns_cfg s)
{
	const int lmax = s->lmax, mmax = s->mmax, mres = s->mres;
	s->stdt_lo.assign(s->vtot, 0.0); s->stdt_hi.assign(s->vtot, 0.0);
	s->van_lo.assign(s->vtot, 0.0); s->van_hi.assign(s->vtot, 0.0);
	for (int im = 0; im <= mmax; im++) {
		const int m = im * mres;
		const int vo = s->voff_h[im];
		for (int l = m; l <= lmax + 1; l++) {
			double ct_lo = 0.0, ct_hi = 0.0;
			if (l > m) ct_lo = 1.0 / alm_a(s, im, l);
			if (s->base_norm == sht_schmidt) {
				if (l < lmax) ct_hi = -alm_b(s, im, l + 2) / alm_a(s, im, l + 2);
				else if (l == lmax) ct_hi = std::sqrt((double)(l + 1 + m) * (double)(l + 1 - m)) / (2 * (l + 1) + 1);
			} else {
				if (l <= lmax) ct_hi = 1.0 / alm_a(s, im, l + 1);
			}
			const int j = l - m;
			s->stdt_lo[vo + j] = (l - 1) * ct_lo;
			s->stdt_hi[vo + j] = -(l + 2) * ct_hi;
			s->van_lo[vo + j] = (l + 1) * ct_lo;
			s->van_hi[vo + j] = -l * ct_hi;
		}
	}
	s->l_2.assign(lmax + 2, 0.0);
	for (int l = 1; l <= lmax + 1; l++) s->l_2[l] = 1.0 / ((double) l * (l + 1));
}

// max over l of |P_l^m(x)| (classic recurrence in long double: its exponent
// range covers every seed below degree 16384)
static double max_plm(shtns_cfg s, int im, long double x, long double sint)
{
	const int m = im * s->mres;
	long double y0 = s->alm[s->alm_off[im]];
	long double sp = 1.0L;
	for (int k = 0; k < m; k++) sp *= sint;
	y0 *= sp;
	long double v = std::fabs(y0);
	if (m + 1 > s->lmax) return (double) v;
	long double y1 = alm_a(s, im, m + 1) * x * y0;
	if (std::fabs(y1) > v) v = std::fabs(y1);
	for (int l = m + 2; l <= s->lmax; l++) {
		long double y2 = alm_a(s, im, l) * x * y1 + alm_b(s, im, l) * y0;
		y0 = y1; y1 = y2;
		if (std::fabs(y1) > v) v = std::fabs(y1);
	}
	return (double) v;
}

static int fft_factorize(int n, std::vector<int>& f)
{
	const int n0 = n;
	f.clear();
	while (n % 8 == 0) { f.push_back(8); n /= 8; }
	while (n % 4 == 0) { f.push_back(4); n /= 4; }
	while (n % 2 == 0) { f.push_back(2); n /= 2; }
	while (n % 3 == 0) { f.push_back(3); n /= 3; }
	while (n % 5 == 0) { f.push_back(5); n /= 5; }
	while (n % 7 == 0) { f.push_back(7); n /= 7; }
	int rmin = 8;
	for (int r : f) rmin = r < rmin ? r : rmin;
	(void) rmin;
	// one CTA holds two padded buffers of a latitude pair in shared memory
	return n == 1 && (int) f.size() <= FFT_MAX_FACTORS && (fft_smem_bytes(n0, 1) <= 227 * 1024 || fft_fused_available(n0));
}

// first checkpoint segment of every order for the current spacing s->ckseg
static void checkpoint_offsets(shtns_cfg s)
{
	s->ckoff_h.assign(s->mmax + 1, 0);
	s->segtot = 0;
	for (int im = 0; im <= s->mmax; im++) {
		s->ckoff_h[im] = (int) s->segtot;
		s->segtot += (s->kmax_h[im] + s->ckseg - 1) / s->ckseg;
	}
}

// ---------------------------------------------------------------------------
static void free_device(shtns_cfg s)
{
	if (s->is_clone) {
		// clones own only their work buffers and streams
	} else {
		void* ptrs[] = {s->d_x, s->d_c, s->d_ck, s->d_tw, s->d_mint, s->d_tw4};
		for (void* p : ptrs) if (p) cudaFree(p);
	}
	free_split(s);
	free_ftab(s);
	if (s->d_alm) cudaFree(s->d_alm);
	if (s->d_loc) cudaFree(s->d_loc);
	s->d_alm = nullptr; s->d_almoff = nullptr; s->d_loc = nullptr; s->loc_cap = 0;
	if (s->d_qq) cudaFree(s->d_qq);
	if (s->d_F) cudaFree(s->d_F);
	if (s->d_stage) cudaFree(s->d_stage);
	if (s->d_fscr) cudaFree(s->d_fscr);
	s->d_fscr = nullptr; s->fscr_cap = 0; s->d_tw4 = nullptr;
	if (s->own_xfer && s->xfer_stream) cudaStreamDestroy(s->xfer_stream);
	if (s->d2h_stream) cudaStreamDestroy(s->d2h_stream);
	for (cudaEvent_t e : s->xev) cudaEventDestroy(e);
	s->d2h_stream = nullptr; s->xev.clear();
	s->d_x = s->d_x2 = s->d_s = s->d_sinv = s->d_w = nullptr;
	s->d_c = s->d_xs = s->d_xa = nullptr;
	s->d_stdt_lo = s->d_stdt_hi = s->d_van_lo = s->d_van_hi = s->d_l2 = nullptr;
	s->d_ck = nullptr; s->d_tw = nullptr; s->d_mint = nullptr;
	s->d_qq = nullptr; s->qq_cap = 0; s->d_F = nullptr; s->F_cap = 0;
	s->d_stage = nullptr; s->stage_cap = 0;
	s->xfer_stream = nullptr; s->own_xfer = 0;
	s->table_bytes = 0;
}

void fft_set_smem_limits();
void shtb_timing_release(shtns_cfg s);

// Upload tables and build the checkpoints.  Returns 0 on success.
static int init_device(shtns_cfg s)
{
	cudaGetDevice(&s->dev);
	static int smem_done[64] = {0};
	if (s->dev >= 0 && s->dev < 64 && !smem_done[s->dev]) { fft_set_smem_limits(); smem_done[s->dev] = 1; }
	const int n2 = s->nlat_2;
	const int nm = s->mmax + 1;
	// grid tables: x, x2, s, 1/s, w (each n2)
	std::vector<double> g(5 * (size_t) n2);
	const double wbase = (s->base_norm == sht_orthonormal) ? 2.0 * M_PI : 0.5;
	for (int t = 0; t < n2; t++) {
		const double x = std::fabs(s->ct_v[s->south_first ? s->nlat - 1 - t : t]);
		const double st = s->st_v[t];
		g[t] = x; g[n2 + t] = x * x; g[2 * n2 + t] = st; g[3 * n2 + t] = 1.0 / st;
		g[4 * n2 + t] = s->wq[t] * wbase;
	}
	// coefficient tables: c | xs | xa | stdt_lo | stdt_hi | van_lo | van_hi | l_2
	const size_t nc = s->ctot + 2 * s->xtot + 4 * s->vtot + (s->lmax + 2);
	std::vector<double> c(nc);
	size_t o = 0;
	auto put = [&](const std::vector<double>& v) { memcpy(c.data() + o, v.data(), sizeof(double) * v.size()); o += v.size(); };
	put(s->ish_c); put(s->ish_xs); put(s->ish_xa); put(s->stdt_lo); put(s->stdt_hi); put(s->van_lo); put(s->van_hi); put(s->l_2);
	// per-order ints
	std::vector<int> mi(6 * (size_t) nm);
	for (int im = 0; im < nm; im++) {
		mi[im] = s->koff_h[im]; mi[nm + im] = s->coff_h[im]; mi[2 * nm + im] = s->xoff_h[im];
		mi[3 * nm + im] = s->voff_h[im]; mi[4 * nm + im] = s->ckoff_h[im]; mi[5 * nm + im] = s->tm_h[im];
	}
	// twiddles exp(+2 pi i j / nphi)
	std::vector<double2> tw(s->nphi);
	for (unsigned j = 0; j < s->nphi; j++) {
		long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double) j / (long double) s->nphi;
		tw[j] = make_double2((double) std::cos(a), (double) std::sin(a));
	}
	const size_t ck_elems = (size_t) s->segtot * n2;
	bool ok = true;
	ok &= shtb_cuda_ok(cudaMalloc(&s->d_x, sizeof(double) * g.size()), "grid tables");
	ok &= ok && shtb_cuda_ok(cudaMalloc(&s->d_c, sizeof(double) * nc), "coefficient tables");
	ok &= ok && shtb_cuda_ok(cudaMalloc(&s->d_mint, sizeof(int) * mi.size()), "order tables");
	ok &= ok && shtb_cuda_ok(cudaMalloc(&s->d_tw, sizeof(double2) * tw.size()), "twiddles");
	ok &= ok && shtb_cuda_ok(cudaMalloc(&s->d_ck, sizeof(double2) * ck_elems), "checkpoints");
	if (ok && s->nphi == 12288) {
		// factor tables of the four-step FFT, 12288 = 96 x 128
		std::vector<double2> t4(96 + 128);
		for (int j = 0; j < 96; j++) {
			long double a = 2.0L * 3.14159265358979323846264338327950288L * j / 96.0L;
			t4[j] = make_double2((double) std::cos(a), (double) std::sin(a));
		}
		for (int j = 0; j < 128; j++) {
			long double a = 2.0L * 3.14159265358979323846264338327950288L * j / 128.0L;
			t4[96 + j] = make_double2((double) std::cos(a), (double) std::sin(a));
		}
		ok &= shtb_cuda_ok(cudaMalloc(&s->d_tw4, sizeof(double2) * t4.size()), "FFT factor tables");
		if (ok) cudaMemcpy(s->d_tw4, t4.data(), sizeof(double2) * t4.size(), cudaMemcpyHostToDevice);
	}
	if (!ok) { free_device(s); return -1; }
	s->table_bytes = sizeof(double) * (g.size() + nc) + sizeof(int) * mi.size() + sizeof(double2) * (tw.size() + ck_elems);
	cudaMemcpy(s->d_x, g.data(), sizeof(double) * g.size(), cudaMemcpyHostToDevice);
	cudaMemcpy(s->d_c, c.data(), sizeof(double) * nc, cudaMemcpyHostToDevice);
	cudaMemcpy(s->d_mint, mi.data(), sizeof(int) * mi.size(), cudaMemcpyHostToDevice);
	cudaMemcpy(s->d_tw, tw.data(), sizeof(double2) * tw.size(), cudaMemcpyHostToDevice);
	s->d_x2 = s->d_x + n2; s->d_s = s->d_x + 2 * n2; s->d_sinv = s->d_x + 3 * n2; s->d_w = s->d_x + 4 * n2;
	double* cp = s->d_c;
	s->d_xs = cp + s->ctot;
	s->d_xa = s->d_xs + s->xtot;
	s->d_stdt_lo = s->d_xa + s->xtot;
	s->d_stdt_hi = s->d_stdt_lo + s->vtot;
	s->d_van_lo = s->d_stdt_hi + s->vtot;
	s->d_van_hi = s->d_van_lo + s->vtot;
	s->d_l2 = s->d_van_hi + s->vtot;
	s->mt.koff = s->d_mint; s->mt.coff = s->d_mint + nm; s->mt.xoff = s->d_mint + 2 * nm;
	s->mt.voff = s->d_mint + 3 * nm; s->mt.ckoff = s->d_mint + 4 * nm; s->mt.tm = s->d_mint + 5 * nm;
	if (!s->xfer_stream) {
		if (cudaStreamCreateWithFlags(&s->xfer_stream, cudaStreamNonBlocking) == cudaSuccess) s->own_xfer = 1;
	}
	launch_checkpoints(s, 0);
	if (!shtb_cuda_ok(cudaDeviceSynchronize(), "plan initialisation")) { free_device(s); return -1; }
	return 0;
}

// ---------------------------------------------------------------------------
extern "C" shtns_cfg shtns_create(int lmax, int mmax, int mres, enum shtns_norm norm)
{
	if (lmax < 2) { plan_error("lmax must be at least 2"); return nullptr; }
	if (lmax > 65534) { plan_error("lmax too large"); return nullptr; }
	if (mres <= 0) { plan_error("MRES must be > 0"); return nullptr; }
	if (mmax < 0 || mmax * mres > lmax) { plan_error("MMAX*MRES should not exceed LMAX"); return nullptr; }
	const int base = ((int) norm) & 0xFF;
	if (base > sht_schmidt) { plan_error("unsupported normalisation"); return nullptr; }
	shtns_cfg s = new shtns_info();
	s->norm_flags = (int) norm;
	s->base_norm = base;
	s->cs_phase = (norm & SHT_NO_CS_PHASE) ? 0 : 1;
	s->mpos_renorm = (norm & SHT_REAL_NORM) ? 0.5 : 1.0;
	s->lmax = lmax; s->mmax = mmax; s->mres = mres;
	s->nlm = (unsigned) nlm_calc(lmax, mmax, mres);
	s->nlm_cplx = 2 * s->nlm - (lmax + 1);
	s->li_v.resize(s->nlm); s->mi_v.resize(s->nlm);
	long lm = 0;
	for (int im = 0; im <= mmax; im++)
		for (int l = im * mres; l <= lmax; l++) { s->li_v[lm] = l; s->mi_v[lm] = im * mres; lm++; }
	s->li = s->li_v.data(); s->mi = s->mi_v.data();
	s->batch = 1; s->spec_dist = s->nlm; s->spat_dist = 0;
	s->dev = -1;
	legendre_tables(s);
	ishioka_tables(s);
	vector_tables(s);
	switch (base) {
		case sht_schmidt: s->Y00_1 = 1.0; s->Y10_ct = 1.0; break;
		case sht_fourpi: s->Y00_1 = 1.0; s->Y10_ct = std::sqrt(1.0 / 3.0); break;
		default: s->Y00_1 = std::sqrt(4.0 * M_PI); s->Y10_ct = std::sqrt(4.0 * M_PI / 3.0);
	}
	s->Y11_st = s->Y10_ct * std::sqrt(0.5 / s->mpos_renorm);
	if (s->cs_phase) s->Y11_st = -s->Y11_st;
	std::lock_guard<std::mutex> lk(g_plans_mu);
	g_plans.push_back(s);
	return s;
}

extern "C" void shtns_unset_grid(shtns_cfg s)
{
	if (!s) return;
	if (!s->is_clone) free_device(s);
	s->grid_set = 0;
	s->nlat = 0; s->nlat_2 = 0; s->nphi = 0; s->nspat = 0;
	s->ct = nullptr; s->st = nullptr;
}

extern "C" int shtns_set_grid_auto(shtns_cfg s, enum shtns_type flags, double eps, int nl_order, int* nlat, int* nphi)
{
	if (!s) { plan_error("null plan"); return -1; }
	const int type = flags & 255;
	const int layout = flags & 0xFFFF00;
	if (type == sht_reg_fast || type == sht_reg_dct || type == sht_reg_poles) {
		plan_error("regular grids are not provided by shtns_b200 (Gauss grids only)");
		return -1;
	}
	if (nl_order <= 0) nl_order = 1;
	if (*nphi == 0) {
		int n = (nl_order + 1) * s->mmax + 1;
		std::vector<int> f;
		while (!fft_factorize(n, f)) n++;
		*nphi = n;
	}
	if (*nlat == 0) {
		int n = ((nl_order + 1) * s->lmax) / 2 + 1;
		n += (n & 1);
		*nlat = n;
	}
	const int nl = *nlat, np = *nphi;
	if (nl & 1) { plan_error("odd nlat is not supported by shtns_b200"); return -1; }
	if (nl <= s->lmax) { plan_error("Nlat must be larger than Lmax"); return -1; }
	if (np <= 2 * s->mmax) { plan_error("the sampling condition Nphi > 2*Mmax is not met."); return -1; }
	if (nl > 65534 || np > 65534) { plan_error("Nlat or Nphi too large"); return -1; }
	std::vector<int> rad;
	if (!fft_factorize(np, rad)) { plan_error("Nphi must factor into 2, 3, 5 and 7 and not exceed 6400 (or be 3*2^k up to 12288)"); return -1; }
	if (layout & SHT_PHI_CONTIGUOUS && layout & SHT_THETA_CONTIGUOUS) { plan_error("conflicting layout flags"); return -1; }
	shtns_unset_grid(s);
	s->fft_radix = rad;
	s->nlat = nl; s->nlat_2 = nl / 2; s->nphi = np;
	s->nspat = (unsigned)((long) nl * np);
	s->nlat_padded = nl;
	s->layout = layout;
	s->phi_contiguous = (layout & SHT_PHI_CONTIGUOUS) ? 1 : 0;
	s->south_first = (layout & SHT_SOUTH_POLE_FIRST) ? 1 : 0;
	s->eps = eps;
	// Gauss grid, generated on the GPU (sht_gauss.cu): nodes and weights
	// refined in double-double and rounded to FP64; sin(theta) is that of the
	// node as rounded to FP64, not of the extended-precision node, so every
	// table describes the same point.  Near the poles an inconsistent pair is
	// amplified (|d sin / sin| = x |dx| / sin^2: 4e-10 at the first row of a
	// 6144-point grid), which would scale the m >= 1 terms.
	std::vector<double> xg, sg, wg;
	if (!gauss_grid_gpu(nl, xg, sg, wg)) { plan_error("Gauss grid generation failed: " + g_last_error); return -1; }
	s->ct_v.assign(nl, 0.0); s->st_v.assign(nl, 0.0);
	s->wq.assign(s->nlat_2, 0.0);
	const double latdir = s->south_first ? -1.0 : 1.0;
	for (int t = 0; t < s->nlat_2; t++) {
		s->ct_v[t] = latdir * xg[t];
		s->ct_v[nl - 1 - t] = -latdir * xg[t];
		s->st_v[t] = sg[t]; s->st_v[nl - 1 - t] = sg[t];
		s->wq[t] = wg[t];
	}
	s->ct = s->ct_v.data(); s->st = s->st_v.data();
	// polar threshold (sht_init.c:522-557): tm[im] = first north row with max_l |P_lm| >= eps
	s->tm_h.assign(s->mmax + 1, 0);
	if (eps > 0.0) {
		for (int im = 1; im <= s->mmax; im++) {
			int it = s->tm_h[im - 1] - 1;
			double v;
			do {
				it++;
				if (it >= s->nlat_2) break;
				v = max_plm(s, im, (long double) xg[it], (long double) sg[it]);
			} while (v < eps);
			s->tm_h[im] = it < s->nlat_2 ? it : s->nlat_2;
		}
	}
	// recurrence checkpoints every 8 degree-pairs when they take at most
	// 512 MB (all threads of a CTA then generate its Y tile in parallel),
	// else every 16 or 32
	for (s->ckseg = 8; s->ckseg < LG_SEG; s->ckseg *= 2) {
		long segs = 0;
		for (int im = 0; im <= s->mmax; im++) segs += (s->kmax_h[im] + s->ckseg - 1) / s->ckseg;
		if ((double) segs * s->nlat_2 * 16.0 <= 512.0 * 1024 * 1024) break;
	}
	checkpoint_offsets(s);
	if (init_device(s) != 0) { plan_error("GPU initialisation failed: " + g_last_error); return -1; }
	s->grid_set = 1;
	if (s->spat_dist < (long) s->nspat) s->spat_dist = s->nspat;
	return (int) s->nspat;
}

extern "C" int shtns_set_grid(shtns_cfg s, enum shtns_type flags, double eps, int nlat, int nphi)
{
	if (nlat == 0 || nphi == 0) { plan_error("nlat or nphi is zero !"); return -1; }
	return shtns_set_grid_auto(s, flags, eps, 0, &nlat, &nphi);
}

extern "C" shtns_cfg shtns_init(enum shtns_type flags, int lmax, int mmax, int mres, int nlat, int nphi)
{
	shtns_cfg s = shtns_create(lmax, mmax, mres, sht_orthonormal);
	if (s && shtns_set_grid(s, flags, 1.e-10, nlat, nphi) < 0) { shtns_destroy(s); return nullptr; }
	return s;
}

static void destroy_plan(shtns_cfg s)
{
	shtb_timing_release(s);
	if (s->is_clone) {
		free_device(s);
		if (s->base) s->base->nclones--;
	} else {
		free_device(s);
	}
	delete s;
}

extern "C" void shtns_destroy(shtns_cfg s)
{
	if (!s) return;
	{
		std::lock_guard<std::mutex> lk(g_plans_mu);
		for (size_t i = 0; i < g_plans.size(); i++)
			if (g_plans[i] == s) { g_plans.erase(g_plans.begin() + i); break; }
	}
	destroy_plan(s);
}

extern "C" void shtns_reset(void)
{
	std::vector<shtns_cfg> all;
	{
		std::lock_guard<std::mutex> lk(g_plans_mu);
		all.swap(g_plans);
	}
	// clones first: they borrow their base plan's tables
	for (shtns_cfg s : all) if (s->is_clone) destroy_plan(s);
	for (shtns_cfg s : all) if (!s->is_clone) destroy_plan(s);
}

extern "C" shtns_cfg shtns_create_with_grid(shtns_cfg base, int mmax, int nofft)
{
	(void) nofft;
	if (!base || mmax != base->mmax) { plan_error("shtns_create_with_grid: only the same mmax is supported"); return nullptr; }
	return cushtns_clone(base, 0, 0);
}

extern "C" void shtns_robert_form(shtns_cfg s, int robert) { if (s) s->robert = robert ? 1 : 0; }

extern "C" void* shtns_malloc(size_t bytes)
{
	void* p = nullptr;
	if (cudaMallocHost(&p, bytes) != cudaSuccess) return nullptr;
	return p;
}
extern "C" void shtns_free(void* p) { if (p) cudaFreeHost(p); }

extern "C" double sh00_1(shtns_cfg s) { return s->Y00_1; }
extern "C" double sh10_ct(shtns_cfg s) { return s->Y10_ct; }
extern "C" double sh11_st(shtns_cfg s) { return s->Y11_st; }
extern "C" double shlm_e1(shtns_cfg s, int l, int m)
{
	double x = s->Y00_1 / std::sqrt(4.0 * M_PI);
	if (s->base_norm == sht_schmidt) x *= std::sqrt(2 * l + 1.0);
	if (m != 0 && s->mpos_renorm == 1.0) x *= std::sqrt(0.5);
	return x;
}

extern "C" int shtns_gauss_wts(shtns_cfg s, double* wts)
{
	if (!s || !s->grid_set) return 0;
	for (int i = 0; i < s->nlat_2; i++) wts[i] = s->wq[i];
	return s->nlat_2;
}

extern "C" void shtns_print_cfg(shtns_cfg s)
{
	printf("Lmax=%d, Mmax*Mres=%d, Mres=%d, Nlm=%d  [GPU %d, norm=%d]\n", s->lmax, s->mmax * s->mres, s->mres, s->nlm, s->dev, s->base_norm);
	if (s->grid_set) printf("Gauss grid : Nlat=%d, Nphi=%d, layout=%s\n", s->nlat, s->nphi, s->phi_contiguous ? "phi-contiguous" : "theta-contiguous");
}

extern "C" int shtns_b200_device(shtns_cfg s) { return s ? s->dev : -1; }
extern "C" size_t shtns_b200_device_bytes(shtns_cfg s)
{
	if (!s) return 0;
	// tables owned by the original plan (recurrence tables, FP64 and INT8
	// Legendre tables), then the plan's own work buffers
	const size_t tables = s->is_clone ? 0 : s->table_bytes + s->ftab_bytes + s->ptab_bytes;
	return tables + sizeof(double) * s->qq_cap + sizeof(double2) * s->F_cap + s->stage_cap + s->fscr_cap + s->pbs_cap +
	       s->pexp_cap + s->bsl_cap + s->bexp_cap;
}

// ---------------------------------------------------------------------------
// Clones share the tables of their base plan and own their work buffers and
// streams (cushtns_clone, sht_gpu.cu:357-370).
extern "C" shtns_cfg cushtns_clone(shtns_cfg b, cudaStream_t compute_stream, cudaStream_t transfer_stream)
{
	if (!b || !b->grid_set) { plan_error("cushtns_clone: plan has no grid"); return nullptr; }
	shtns_cfg s = new shtns_info();
	// copy everything (host tables are duplicated, device tables shared)
	*s = *b;
	s->li = s->li_v.data(); s->mi = s->mi_v.data();
	s->ct = s->ct_v.data(); s->st = s->st_v.data();
	s->is_clone = 1;
	s->base = b->is_clone ? b->base : b;
	s->base->nclones++;
	s->d_qq = nullptr; s->qq_cap = 0; s->d_F = nullptr; s->F_cap = 0;
	s->d_stage = nullptr; s->stage_cap = 0;
	s->d_fscr = nullptr; s->fscr_cap = 0;
	s->d_alm = nullptr; s->d_almoff = nullptr; s->d_loc = nullptr; s->loc_cap = 0;
	s->d_yexp = nullptr; s->d_boff = nullptr; s->split_chunks = 0; s->split_kc = 0;
	s->d_bsl = nullptr; s->bsl_cap = 0; s->d_bexp = nullptr; s->bexp_cap = 0; s->d_split_err = nullptr;
	s->d_ptab = nullptr; s->ptab_bytes = 0; s->ptab_ns = 0; s->d_ptoff = nullptr; s->d_pkoff = nullptr;
	s->d_pvoff = nullptr; s->d_pt0 = nullptr; s->d_pkf = nullptr; s->ptab_kblocks = 0; s->ptab_ttiles = 0;
	s->d_pbs = nullptr; s->pbs_cap = 0; s->d_pexp = nullptr; s->pexp_cap = 0;
	s->d_ftab = nullptr; s->ftab_bytes = 0; s->d_ftoff = nullptr; s->d_ftb0 = nullptr; s->d_fzero = nullptr;
	s->ftab_failed = 0;
	s->xfer_stream = nullptr; s->own_xfer = 0;
	s->d2h_stream = nullptr; s->xev.clear();
	s->ev.clear(); s->ev_stage.clear(); s->ev_used = 0; s->timing = 0;
	cushtns_set_streams(s, compute_stream, transfer_stream);
	std::lock_guard<std::mutex> lk(g_plans_mu);
	g_plans.push_back(s);
	return s;
}

extern "C" int cushtns_init_gpu(shtns_cfg s)
{
	if (!s || !s->grid_set) return -1;
	return s->dev;
}

extern "C" void cushtns_set_streams(shtns_cfg s, cudaStream_t compute_stream, cudaStream_t transfer_stream)
{
	if (!s) return;
	s->comp_stream = compute_stream;
	if (transfer_stream) {
		if (s->own_xfer && s->xfer_stream) cudaStreamDestroy(s->xfer_stream);
		s->xfer_stream = transfer_stream;
		s->own_xfer = 0;
	} else if (!s->xfer_stream) {
		if (cudaStreamCreateWithFlags(&s->xfer_stream, cudaStreamNonBlocking) == cudaSuccess) s->own_xfer = 1;
	}
}

// ---------------------------------------------------------------------------
// Per-stage timing: a pool of event pairs recorded on the compute stream,
// read back only when the caller asks (or when the pool is full).
static void timing_collect(shtns_cfg s)
{
	for (int i = 0; i < s->ev_used; i++) {
		float ms = 0.f;
		cudaEventSynchronize(s->ev[2 * i + 1]);
		if (cudaEventElapsedTime(&ms, s->ev[2 * i], s->ev[2 * i + 1]) == cudaSuccess) {
			s->stage_ms[s->ev_stage[i]] += ms;
			s->stage_calls[s->ev_stage[i]]++;
		}
	}
	s->ev_used = 0;
}

void shtb_timing_release(shtns_cfg s)
{
	for (cudaEvent_t e : s->ev) cudaEventDestroy(e);
	s->ev.clear(); s->ev_stage.clear(); s->ev_used = 0;
}

void shtb_stage_begin(shtns_cfg s, int stage)
{
	if (!s->timing) return;
	const int pool = 256;
	if (s->ev.empty()) {
		s->ev.resize(2 * pool);
		s->ev_stage.assign(pool, 0);
		for (auto& e : s->ev) cudaEventCreate(&e);
	}
	if (s->ev_used >= pool) timing_collect(s);
	s->ev_stage[s->ev_used] = stage;
	cudaEventRecord(s->ev[2 * s->ev_used], s->comp_stream);
}

void shtb_stage_end(shtns_cfg s)
{
	if (!s->timing) return;
	cudaEventRecord(s->ev[2 * s->ev_used + 1], s->comp_stream);
	s->ev_used++;
}

extern "C" void shtns_b200_set_timing(shtns_cfg s, int on)
{
	if (!s) return;
	if (!on && s->timing) { timing_collect(s); }
	s->timing = on ? 1 : 0;
	if (on) {
		for (int i = 0; i < SHTB_NSTAGES; i++) { s->stage_ms[i] = 0.0; s->stage_calls[i] = 0; }
	}
}

extern "C" int shtns_b200_stage_times(shtns_cfg s, double* ms, long* calls)
{
	if (!s) return -1;
	timing_collect(s);
	for (int i = 0; i < SHTB_NSTAGES; i++) {
		if (ms) ms[i] = s->stage_ms[i];
		if (calls) calls[i] = s->stage_calls[i];
		s->stage_ms[i] = 0.0; s->stage_calls[i] = 0;
	}
	return SHTB_NSTAGES;
}

extern "C" int shtns_b200_polar_rows(shtns_cfg s, int* tm)
{
	if (!s || !s->grid_set) return 0;
	for (int im = 0; im <= s->mmax; im++) tm[im] = s->tm_h[im];
	return s->mmax + 1;
}

// ---------------------------------------------------------------------------
// Tuning options (shtns_b200_set_option).  Checkpoint spacing rebuilds the
// recurrence checkpoint table of the plan (not allowed on clones, which share
// it).
extern "C" int shtns_b200_set_option(shtns_cfg s, int option, int value)
{
	if (!s) return -1;
	switch (option) {
		case 1:   // latitude pairs per FFT CTA
			if (value != 0 && value != 1 && value != 2 && value != 4 && value != 8) return -1;
			s->fft_pairs = value;
			return 0;
		case 5:   // Legendre tile shape: warps along the rows, 8 = SIMT kernels (0 automatic)
			if (value != 0 && value != 1 && value != 2 && value != 4 && value != 8) return -1;
			s->tile_wm = value;
			return 0;
		case 4:   // split-precision synthesis: slices per operand (0 = FP64)
			if (value != 0 && (value < 3 || value > 7)) return -1;
			s->split_ns = value;
			return 0;
		case 2: { // recurrence checkpoint spacing
			if (value != 8 && value != 16 && value != 32) return -1;
			if (!s->grid_set || s->is_clone || s->nclones > 0) return -1;
			if (value == s->ckseg) return 0;
			cudaDeviceSynchronize();
			double2* old = s->d_ck;
			const int old_seg = s->ckseg;
			s->ckseg = value;
			checkpoint_offsets(s);
			double2* nck = nullptr;
			if (cudaMalloc(&nck, sizeof(double2) * (size_t) s->segtot * s->nlat_2) != cudaSuccess) {
				cudaGetLastError();
				s->ckseg = old_seg;
				checkpoint_offsets(s);
				shtb_set_error(3, "out of device memory for checkpoints");
				return -1;
			}
			cudaFree(old);
			s->d_ck = nck;
			free_split(s);          // split-precision and FP64 tables derive from the checkpoints
			free_ftab(s);
			const int nm = s->mmax + 1;
			cudaMemcpy(s->d_mint + 4 * nm, s->ckoff_h.data(), sizeof(int) * nm, cudaMemcpyHostToDevice);
			launch_checkpoints(s, 0);
			return shtb_cuda_ok(cudaDeviceSynchronize(), "checkpoint rebuild") ? 0 : -1;
		}
		case 3:   // FFT kernels: 0 automatic, 1 generic mixed-radix, 2 fused without prefetch,
		          // 3 prefetched loads with per-thread stores
			if (value < 0 || value > 3) return -1;
			s->fft_generic = value;
			return 0;
		case 7:   // test hook: bytes the prefetching FFT kernels wait for beyond their tensor copies, 0..4096
		          // (a positive value makes their bounded wait give up: error-path tests)
			if (value < 0 || value > 4096 || (value & 15)) return -1;
			s->fft_extra_tx = value;
			return 0;
		case 8:   // split-precision form: 0 precomputed int8 digit table (synthesis and analysis), 1 on-the-fly FP16 (synthesis)
			if (value != 0 && value != 1) return -1;
			s->split_form = value;
			return 0;
		case 9:   // test hook: fill the no-allocation entry point's static scratch with this byte
			if (value < 0 || value > 255) return -1;
			return shtb_noalloc_fill(value);
		case 10:  // FP64 Legendre values: 0 automatic (precomputed table within a memory budget), 1 on the fly, 2 table
			if (value < 0 || value > 2) return -1;
			s->ftab_mode = value;
			s->ftab_failed = 0;
			return 0;
		default:
			return -1;
	}
}

extern "C" int shtns_b200_get_option(shtns_cfg s, int option)
{
	if (!s) return -1;
	switch (option) {
		case 1: return s->fft_pairs;
		case 2: return s->ckseg;
		case 3: return s->fft_generic;
		case 4: return s->split_ns;
		case 5: return s->tile_wm;
		case 6: return fft_last_path();   // FFT kernels of the last launch in this process
		case 7: return s->fft_extra_tx;
		case 8: return s->split_form;
		case 10: return s->ftab_mode;
		default: return -1;
	}
}
