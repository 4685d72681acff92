// Rotations of spherical-harmonic expansions on sm_100a (shtns.h:186-218;
// sht_func.c:37-53 and 1380-2200).
//
// A rotation with Euler angles (alpha, beta, gamma) in the intrinsic ZYZ
// convention acts on the coefficients of degree l as
//   R_m' = e^{-i m' gamma} sum_m d^l_{m'm}(beta) e^{-i m alpha} Q_m,
// an active rotation of the field (checked against point values).  The
// Wigner d-matrices follow Gumerov and Duraiswami's recursion
// (arXiv:1403.7698), as the reference does: row m' = 0 is
// d_{0m} = P~_l^m(cos beta) (Schmidt semi-normalised, no Condon-Shortley
// phase, eq. 32), row 1 comes from P~_{l+1} (eq. 105), row -1 and rows
// +-m', m' >= 2, from the two previous rows of the same sign (eqs. 106, 108),
// always for columns m >= |m'| (a quarter of the matrix); the other entries
// follow from d_{m'm} = d_{-m,-m'} = (-1)^{m-m'} d_{mm'} = (-1)^{m-m'} d_{-m',-m}.
//
// GPU layout: one CTA per degree l.  Threads own columns m (and -m); the
// quarter rows are built in shared memory one pair (m', -m') per step, and
// each element is applied at once through the symmetries: contributions to
// the outputs indexed by the column stay in the owner's registers, those
// indexed by the row are summed over the CTA (warp shuffles, then one warp)
// and stored once per step.  The matrices are never stored.
#include "sht_internal.h"

#include <cmath>
#include <cstring>
#include <vector>

#define ROT_STREAMS_DECL 4

struct shtns_rot_ {
	int lmax, mmax;
	int norm;
	double no_cs_phase;      // -1 without Condon-Shortley phase (rotating beta's sign)
	double m0_renorm;        // sqrt(2) with SHT_REAL_NORM
	double alpha, beta, gamma, cos_beta, sin_beta;
	int flag_ag;             // bit 0: alpha != 0, bit 1: gamma != 0
	shtns_cfg leg;           // lmax+1, Schmidt, no CS phase: tables for P~_n^m(cos beta)
	double* d_plm;           // P~_n^m, m, n <= lmax+1, [ofs(m) + n - m]
	double2* d_e;            // e^{-i m alpha} (m <= lmax), then e^{-i m gamma}
	void* d_buf; size_t buf_cap;
	int ready;               // angles set
	cudaStream_t side[ROT_STREAMS_DECL];   // degree groups run concurrently on these
	cudaEvent_t ev[ROT_STREAMS_DECL + 1];
};

void launch_plm_table(shtns_cfg s, double x, double st, double* out, cudaStream_t st_);

namespace {

struct RotParams {
	int lmax, mmax, L1;      // L1 = lmax + 1: degrees of the P~ table
	int cplx;                // 0: real field, LM layout (mres 1); 1: complex field, LM_cplx layout
	double cos_beta, sin_beta, m0_renorm;
	const double* plm;
	const double2 *ea, *eg;
	const double2* Q;
	double2* R;
	double2* acc;            // row-type sums, degree l at offset l^2 (index m + l)
	int l0, l1;              // degrees of this launch
	double* wig;             // Wigner matrix output (one degree) instead of applying, or null
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cax(double a, double2 z, double2 acc) { return make_double2(fma(a, z.x, acc.x), fma(a, z.y, acc.y)); }

__device__ __forceinline__ double plmv(const RotParams& p, int m, int n)
{
	return p.plm[(long) m * (p.L1 + 2) - (long) m * (m + 1) / 2 + (n - m)];
}

__device__ __forceinline__ double clm(int l, int m) { return (m < l) ? sqrt((double)((l - m) * (l + m + 1))) : 0.0; }

// pre-rotated input Q'_m = e^{-i m alpha} Q_m, m in [-l, l]
__device__ double2 qin(const RotParams& p, int l, int m)
{
	const int am = m < 0 ? -m : m;
	if (am > p.mmax || am > l) return make_double2(0.0, 0.0);
	if (!p.cplx) {
		double2 z = p.Q[(long) am * (2 * p.lmax + 1 - am) / 2 + l];
		if (am == 0) return make_double2(z.x * p.m0_renorm, 0.0);
		z = cmul(z, p.ea[am]);
		if (m < 0) { z = cconj(z); if (am & 1) z = make_double2(-z.x, -z.y); }    // Q_{-m} = (-1)^m conj(Q_m)
		return z;
	}
	const long ll = (l <= p.mmax) ? (long) l * (l + 1) : (long) p.mmax * (2 * l - p.mmax) + l;
	const double2 z = p.Q[ll + m];
	return m > 0 ? cmul(z, p.ea[m]) : (m < 0 ? cmul(z, cconj(p.ea[-m])) : z);
}

// quarter element x = d(a, b), b >= |a|: row-type sums (R_a, R_-a), column sums (R_b, R_-b)
#define ROT_NT 256                 // threads per CTA at most (two CTAs per SM at 128 registers)
#define ROT_LMAX 2047              // 8 columns per thread at most

template <int KC>
__device__ __forceinline__ void apply_elem(int a, int b, int k, double x, double2 qa, double2 qma, const double2 (&qp)[KC],
                                           const double2 (&qm)[KC], double2 (&cp)[KC], double2 (&cn)[KC], double2& sa, double2& sma)
{
	const int aa = a < 0 ? -a : a;
	const double px = ((b - a) & 1) ? -x : x;
	sa = cax(x, qp[k], sa);                               // (a, b)
	if (b > aa) {
		cn[k] = cax(x, qma, cn[k]);                       // (-b, -a)
		cp[k] = cax(px, qa, cp[k]);                       // (b, a)
		sma = cax(px, qm[k], sma);                        // (-a, -b)
	} else if (a > 0) {
		cn[k] = cax(x, qma, cn[k]);                       // b = a: (-a, -a)
	} else if (a < 0) {
		cp[k] = cax(x, qa, cp[k]);                        // b = -a: (-a, a)
	}
}

__device__ __forceinline__ void wig_put(const RotParams& p, int l, int a, int b, double x)
{
	const long w = 2 * l + 1;
	const double px = ((b - a) & 1) ? -x : x;
	p.wig[(a + l) * w + (b + l)] = x;
	p.wig[(-b + l) * w + (-a + l)] = x;
	p.wig[(b + l) * w + (a + l)] = px;
	p.wig[(-a + l) * w + (-b + l)] = px;
}

// warp sums of (sa, sma) -> red[slot][warp]
__device__ __forceinline__ void warp_sums(double2 sa, double2 sma, double* red, int lane, int warp)
{
	double v[4] = {sa.x, sa.y, sma.x, sma.y};
	#pragma unroll
	for (int i = 0; i < 4; i++)
		for (int o = 16; o; o >>= 1) v[i] += __shfl_xor_sync(0xffffffffu, v[i], o);
	if (lane == 0) {
		#pragma unroll
		for (int i = 0; i < 4; i++) red[warp * 4 + i] = v[i];
	}
}

// warp 0: total of red[slot] over the warps, stored as the row sums of step a
__device__ __forceinline__ void store_row_sums(const double* red, int nw, int lane, int a, double2* racc, int l)
{
	double v[4] = {0.0, 0.0, 0.0, 0.0};
	if (lane < nw) {
		#pragma unroll
		for (int i = 0; i < 4; i++) v[i] = red[lane * 4 + i];
	}
	#pragma unroll
	for (int i = 0; i < 4; i++)
		for (int o = 16; o; o >>= 1) v[i] += __shfl_xor_sync(0xffffffffu, v[i], o);
	if (lane == 0) {
		if (a == 0) racc[l] = make_double2(v[0] + v[2], v[1] + v[3]);
		else { racc[l + a] = make_double2(v[0], v[1]); racc[l - a] = make_double2(v[2], v[3]); }
	}
}

template <int KC>
__global__ void __launch_bounds__(ROT_NT, KC <= 4 ? 2 : 1) rot_kernel(RotParams p)
{
	extern __shared__ double sm[];
	const int l = p.l1 - blockIdx.x;                 // largest degrees first
	if (l < p.l0 || l < 1) return;
	const int nt = blockDim.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = (nt + 31) >> 5;
	const int W = p.l1 + 2;
	double* P0 = sm;
	double* P1 = sm + W;
	double* N0 = sm + 2 * W;
	double* N1 = sm + 3 * W;
	double* red = sm + 4 * W;                          // [2][32][4]
	double2* racc = p.acc ? p.acc + (long) l * l : nullptr;
	const bool apply = (p.wig == nullptr);
	double2 qp[KC], qm[KC], cp[KC], cn[KC];
	#pragma unroll
	for (int k = 0; k < KC; k++) {
		const int b = tid + k * nt;
		qp[k] = qm[k] = cp[k] = cn[k] = make_double2(0.0, 0.0);
		if (apply && b <= l) { qp[k] = qin(p, l, b); qm[k] = qin(p, l, -b); }
	}
	if (tid == 0) { P0[l + 1] = 0.0; P1[l + 1] = 0.0; N0[l + 1] = 0.0; N1[l + 1] = 0.0; }
	const double d_1 = 1.0 / ((double) l * (l + 1.0));
	const double cbp = (1.0 + p.cos_beta) * 0.5, cbm = (1.0 - p.cos_beta) * 0.5;

	// step 0: rows 0 and 1 (eqs. 32 and 105); row 0 applied
	{
		double2 sa = make_double2(0.0, 0.0), sma = sa;
		const double2 q0 = apply ? qin(p, l, 0) : sa;
		#pragma unroll
		for (int k = 0; k < KC; k++) {
			const int b = tid + k * nt;
			if (b > l) continue;
			const double x0 = plmv(p, b, l);
			P0[b] = x0;
			N0[b] = x0;
			if (b >= 1) {
				const double a = sqrt((double)((l + 1 + b) * (l + 1 - b)) * d_1) * p.sin_beta;
				const double b1 = sqrt((double)((l - b + 1) * (l - b + 2)) * d_1) * cbp;
				const double b2 = sqrt((double)((l + b + 1) * (l + b + 2)) * d_1) * cbm;
				P1[b] = b2 * plmv(p, b + 1, l + 1) + b1 * plmv(p, b - 1, l + 1) + a * plmv(p, b, l + 1);
			}
			if (apply) apply_elem<KC>(0, b, k, x0, q0, q0, qp, qm, cp, cn, sa, sma);
			else wig_put(p, l, 0, b, x0);
		}
		if (apply) warp_sums(sa, sma, red, lane, warp);
	}
	__syncthreads();
	if (apply && warp == 0) store_row_sums(red, nw, lane, 0, racc, l);

	// step 1: row -1 (eq. 108 with m' = -1); rows 1 and -1 applied
	{
		double2 sa = make_double2(0.0, 0.0), sma = sa;
		const double2 q1 = apply ? qin(p, l, 1) : sa, qm1 = apply ? qin(p, l, -1) : sa;
		const double c_1 = 1.0 / clm(l, 0);
		#pragma unroll
		for (int k = 0; k < KC; k++) {
			const int b = tid + k * nt;
			if (b < 1 || b > l) continue;
			const double x1 = P1[b];
			const double xm = x1 + c_1 * (-clm(l, b - 1) * P0[b - 1] + clm(l, b) * P0[b + 1]);
			N1[b] = xm;
			if (apply) {                                   // sa: R_1, sma: R_-1
				apply_elem<KC>(1, b, k, x1, q1, qm1, qp, qm, cp, cn, sa, sma);
				apply_elem<KC>(-1, b, k, xm, qm1, q1, qp, qm, cp, cn, sma, sa);
			} else {
				wig_put(p, l, 1, b, x1);
				wig_put(p, l, -1, b, xm);
			}
		}
		if (apply) warp_sums(sa, sma, red + 128, lane, warp);
	}
	__syncthreads();
	if (apply && warp == 0) store_row_sums(red + 128, nw, lane, 1, racc, l);

	// steps m' = 2..l: rows m' and -m' from the two previous rows of each sign
	double *pp2 = P0, *pp1 = P1, *nn2 = N0, *nn1 = N1;
	for (int mp = 2; mp <= l; mp++) {
		double* rd = red + 128 * (mp & 1);
		double2 sa = make_double2(0.0, 0.0), sma = sa;
		const double2 qa = apply ? qin(p, l, mp) : sa, qma = apply ? qin(p, l, -mp) : sa;
		const double c_1 = 1.0 / clm(l, mp - 1), cmp2 = clm(l, mp - 2);
		#pragma unroll
		for (int k = 0; k < KC; k++) {
			const int b = tid + k * nt;
			if (b < mp || b > l) continue;
			const double cb1 = clm(l, b - 1), cb0 = clm(l, b);
			const double H = (cmp2 * pp2[b] + cb1 * pp1[b - 1] - cb0 * pp1[b + 1]) * c_1;     // eq. 106
			const double Hn = (cmp2 * nn2[b] - cb1 * nn1[b - 1] + cb0 * nn1[b + 1]) * c_1;    // eq. 108
			pp2[b] = H;
			nn2[b] = Hn;
			if (apply) {                                   // sa: R_mp, sma: R_-mp
				apply_elem<KC>(mp, b, k, H, qa, qma, qp, qm, cp, cn, sa, sma);
				apply_elem<KC>(-mp, b, k, Hn, qma, qa, qp, qm, cp, cn, sma, sa);
			} else {
				wig_put(p, l, mp, b, H);
				wig_put(p, l, -mp, b, Hn);
			}
		}
		if (apply) warp_sums(sa, sma, rd, lane, warp);
		__syncthreads();
		if (apply && warp == 0) store_row_sums(rd, nw, lane, mp, racc, l);
		double* t = pp2; pp2 = pp1; pp1 = t;
		t = nn2; nn2 = nn1; nn1 = t;
	}
	if (!apply) return;
	__syncthreads();
	// outputs: row sums + column sums, post-rotation by gamma
	#pragma unroll
	for (int k = 0; k < KC; k++) {
		const int b = tid + k * nt;
		if (b > l || b > p.mmax) continue;
		const double2 rb = make_double2(racc[l + b].x + cp[k].x, racc[l + b].y + cp[k].y);
		const double2 rmb = make_double2(racc[l - b].x + cn[k].x, racc[l - b].y + cn[k].y);
		if (!p.cplx) {
			const long lm = (long) b * (2 * p.lmax + 1 - b) / 2 + l;
			p.R[lm] = (b == 0) ? make_double2(rb.x / p.m0_renorm, 0.0) : cmul(rb, p.eg[b]);
		} else {
			const long ll = (l <= p.mmax) ? (long) l * (l + 1) : (long) p.mmax * (2 * l - p.mmax) + l;
			if (b == 0) p.R[ll] = rb;
			else { p.R[ll + b] = cmul(rb, p.eg[b]); p.R[ll - b] = cmul(rmb, cconj(p.eg[b])); }
		}
	}
}

// degree 0 (invariant), and rotations about z only (beta = 0)
__global__ void rot_z_kernel(RotParams p, int with_l0_only)
{
	const int l = blockIdx.x;
	for (int b = threadIdx.x; b <= l && b <= p.mmax; b += blockDim.x) {
		if (with_l0_only && l > 0) return;
		if (!p.cplx) {
			const long lm = (long) b * (2 * p.lmax + 1 - b) / 2 + l;
			p.R[lm] = (b == 0) ? p.Q[lm] : cmul(p.Q[lm], p.ea[b]);
		} else {
			const long ll = (l <= p.mmax) ? (long) l * (l + 1) : (long) p.mmax * (2 * l - p.mmax) + l;
			if (b == 0) p.R[ll] = p.Q[ll];
			else { p.R[ll + b] = cmul(p.Q[ll + b], p.ea[b]); p.R[ll - b] = cmul(p.Q[ll - b], cconj(p.ea[b])); }
		}
	}
}

// SH_Zrotate: R_lm = Q_lm (cos(m alpha) - i sin(m alpha))
__global__ void zrotate_kernel(const double2* __restrict__ Q, double2* __restrict__ R, int lmax, int mmax, int mres,
                               double alpha)
{
	const int im = blockIdx.y;
	const int m = im * mres;
	const int l = m + blockIdx.x * blockDim.x + threadIdx.x;
	if (l > lmax || im > mmax) return;
	const long lm = (long) im * (2 * lmax + 2 - (im + 1) * mres) / 2 + l;
	double sn, cs;
	sincos((double) m * alpha, &sn, &cs);
	R[lm] = (m == 0) ? Q[lm] : cmul(Q[lm], make_double2(cs, -sn));
}

// cos(phi) + i sin(phi), exact at the angles the reference special-cases
void eiphi(double phi, double& c, double& s)
{
	if (phi == 0.0) { c = 1.0; s = 0.0; }
	else if (phi == M_PI) { c = -1.0; s = 0.0; }
	else if (phi == M_PI / 2) { c = 0.0; s = 1.0; }
	else if (phi == 3 * M_PI / 2 || phi == -M_PI / 2) { c = 0.0; s = -1.0; }
	else if (phi == M_PI / 4) { c = std::sqrt(0.5); s = std::sqrt(0.5); }
	else if (phi == M_PI / 3) { c = 0.5; s = std::sqrt(3.0) * 0.5; }
	else { c = std::cos(phi); s = std::sin(phi); }
}

bool rot_buf(shtns_rot r, size_t bytes)
{
	if (r->buf_cap >= bytes && r->d_buf) return true;
	if (r->d_buf) cudaFree(r->d_buf);
	r->d_buf = nullptr; r->buf_cap = 0;
	if (!shtb_cuda_ok(cudaMalloc(&r->d_buf, bytes), "rotation buffers")) { r->d_buf = nullptr; return false; }
	r->buf_cap = bytes;
	return true;
}

size_t al256(size_t b) { return (b + 255) & ~(size_t) 255; }

template <int KC>
void launch_rot(const RotParams& p, int nt, size_t smem, cudaStream_t st)
{
	cudaFuncSetAttribute(rot_kernel<KC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
	rot_kernel<KC><<<p.l1 - p.l0 + 1, nt, smem, st>>>(p);
}

void launch_rot_group(RotParams p, int l0, int l1, cudaStream_t st)
{
	const int nt = std::min(ROT_NT, (l1 + 1 + 31) / 32 * 32);
	const int kc = (l1 + 1 + nt - 1) / nt;
	const size_t smem = sizeof(double) * (4 * (size_t)(l1 + 2) + 256);
	p.l0 = l0; p.l1 = l1;
	if (kc <= 1) launch_rot<1>(p, nt, smem, st);
	else if (kc <= 2) launch_rot<2>(p, nt, smem, st);
	else if (kc <= 4) launch_rot<4>(p, nt, smem, st);
	else launch_rot<8>(p, nt, smem, st);
	shtb_count_launch();
}

// all degrees 1..lmax, grouped by size (threads and shared memory per
// group); the groups are independent and run concurrently on the side
// streams, largest first, joined back into st
bool run_rotation(shtns_rot r, RotParams p, int lmin, int lmax, cudaStream_t st)
{
	std::vector<std::pair<int, int>> groups;
	for (int l0 = lmin; l0 <= lmax;) {
		int l1 = (l0 < 32) ? 31 : 2 * l0 - 1;
		if (l1 > lmax) l1 = lmax;
		groups.push_back({l0, l1});
		l0 = l1 + 1;
	}
	cudaEventRecord(r->ev[ROT_STREAMS_DECL], st);
	for (int i = 0; i < ROT_STREAMS_DECL; i++) cudaStreamWaitEvent(r->side[i], r->ev[ROT_STREAMS_DECL], 0);
	for (size_t g = groups.size(); g-- > 0;)
		launch_rot_group(p, groups[g].first, groups[g].second, r->side[(groups.size() - 1 - g) % ROT_STREAMS_DECL]);
	for (int i = 0; i < ROT_STREAMS_DECL; i++) {
		cudaEventRecord(r->ev[i], r->side[i]);
		cudaStreamWaitEvent(st, r->ev[i], 0);
	}
	return shtb_cuda_ok(cudaGetLastError(), "rotation launch");
}

RotParams rot_params(shtns_rot r)
{
	RotParams p;
	memset(&p, 0, sizeof(p));
	p.lmax = r->lmax; p.mmax = r->mmax; p.L1 = r->lmax + 1;
	p.cos_beta = r->cos_beta; p.sin_beta = r->sin_beta; p.m0_renorm = r->m0_renorm;
	p.plm = r->d_plm;
	p.ea = r->d_e; p.eg = r->d_e + (r->lmax + 1);
	return p;
}

// host arrays Q (n complex) -> rotation -> R
void rot_apply(shtns_rot r, const cplx* Qh, cplx* Rh, int cplx_field)
{
	if (!r || !Qh || !Rh) { shtb_set_error(1, "rotation: null argument"); return; }
	if (!r->ready) { shtb_set_error(1, "rotation: angles not set"); return; }
	const long n = cplx_field ? (long) nlm_cplx_calc(r->lmax, r->mmax, 1) : (long) nlm_calc(r->lmax, r->mmax, 1);
	const long nacc = (long)(r->lmax + 1) * (r->lmax + 1);
	const size_t qb = al256(sizeof(double2) * n);
	if (!rot_buf(r, 2 * qb + sizeof(double2) * nacc)) return;
	double2* q = static_cast<double2*>(r->d_buf);
	double2* out = reinterpret_cast<double2*>(static_cast<char*>(r->d_buf) + qb);
	double2* acc = reinterpret_cast<double2*>(static_cast<char*>(r->d_buf) + 2 * qb);
	cudaStream_t st = r->leg->comp_stream;
	cudaMemcpyAsync(q, Qh, sizeof(double2) * n, cudaMemcpyHostToDevice, st);
	RotParams p = rot_params(r);
	p.cplx = cplx_field; p.Q = q; p.R = out; p.acc = acc;
	if (r->beta == 0.0) {
		rot_z_kernel<<<r->lmax + 1, 128, 0, st>>>(p, 0);
		shtb_count_launch();
	} else {
		rot_z_kernel<<<1, 32, 0, st>>>(p, 1);               // degree 0 is invariant
		shtb_count_launch();
		if (!run_rotation(r, p, 1, r->lmax, st)) return;
	}
	if (!shtb_cuda_ok(cudaGetLastError(), "rotation launch")) return;
	cudaMemcpyAsync(Rh, out, sizeof(double2) * n, cudaMemcpyDeviceToHost, st);
	shtb_cuda_ok(cudaStreamSynchronize(st), "rotation");
}

} // namespace

// ---------------------------------------------------------------------------
extern "C" shtns_rot shtns_rotation_create(const int lmax, const int mmax, int norm)
{
	if (lmax < 1 || mmax < 0 || mmax > lmax) { shtb_set_error(1, "shtns_rotation_create: invalid lmax/mmax"); return nullptr; }
	if (lmax > ROT_LMAX) { shtb_set_error(1, "shtns_rotation_create: lmax above 2047 is not supported"); return nullptr; }
	shtns_rot r = new shtns_rot_();
	r->lmax = lmax; r->mmax = mmax; r->norm = norm;
	r->no_cs_phase = (norm & SHT_NO_CS_PHASE) ? -1.0 : 1.0;
	r->m0_renorm = (norm & SHT_REAL_NORM) ? std::sqrt(2.0) : 1.0;
	// P~_n^m(cos beta) up to degree and order lmax+1: Schmidt semi-normalised, no CS phase
	r->leg = shtns_create(lmax + 1, lmax + 1, 1, (enum shtns_norm)(sht_schmidt | SHT_NO_CS_PHASE));
	if (!r->leg) { delete r; return nullptr; }
	const long nplm = nlm_calc(lmax + 1, lmax + 1, 1);
	const size_t plm_bytes = (sizeof(double) * nplm + 255) & ~(size_t) 255;     // the double2 table after it stays 16-byte aligned
	void* d = nullptr;
	if (!shtb_cuda_ok(cudaMalloc(&d, plm_bytes + sizeof(double2) * 2 * (lmax + 1)), "rotation tables")) {
		shtns_destroy(r->leg);
		delete r;
		return nullptr;
	}
	r->d_plm = static_cast<double*>(d);
	r->d_e = reinterpret_cast<double2*>(static_cast<char*>(d) + plm_bytes);
	for (int i = 0; i < ROT_STREAMS_DECL; i++) cudaStreamCreateWithFlags(&r->side[i], cudaStreamNonBlocking);
	for (int i = 0; i <= ROT_STREAMS_DECL; i++) cudaEventCreateWithFlags(&r->ev[i], cudaEventDisableTiming);
	return r;
}

extern "C" void shtns_rotation_destroy(shtns_rot r)
{
	if (!r) return;
	for (int i = 0; i < ROT_STREAMS_DECL; i++) if (r->side[i]) cudaStreamDestroy(r->side[i]);
	for (int i = 0; i <= ROT_STREAMS_DECL; i++) if (r->ev[i]) cudaEventDestroy(r->ev[i]);
	if (r->d_plm) cudaFree(r->d_plm);
	if (r->d_buf) cudaFree(r->d_buf);
	if (r->leg) shtns_destroy(r->leg);
	delete r;
}

extern "C" void shtns_rotation_set_angles_ZYZ(shtns_rot r, double alpha, double beta, double gamma)
{
	if (!r) return;
	beta *= r->no_cs_phase;           // the CS phase amounts to a rotation by pi, i.e. beta -> -beta
	if (std::fabs(beta) > M_PI) { shtb_set_error(1, "rotation: angle beta must be between -pi and pi"); return; }
	if (beta < 0.0) {                 // beta < 0: rotate alpha and gamma by pi instead
		alpha = (alpha > 0) ? alpha - M_PI : alpha + M_PI;
		beta = -beta;
		gamma = (gamma > 0) ? gamma - M_PI : gamma + M_PI;
	} else if (beta == 0.0) {
		alpha += gamma;
		gamma = 0.0;
	}
	double cb, sb, ca, sa, cg, sg;
	eiphi(beta, cb, sb);
	eiphi(-alpha, ca, sa);
	eiphi(-gamma, cg, sg);
	r->cos_beta = cb; r->sin_beta = sb;
	r->alpha = alpha; r->beta = beta; r->gamma = gamma;
	r->flag_ag = (alpha != 0) + 2 * (gamma != 0);
	// e^{-i m alpha}, e^{-i m gamma} by repeated products (exact powers at the special angles)
	const int n = r->lmax + 1;
	std::vector<double2> e(2 * n);
	double2 za = make_double2(1.0, 0.0), zg = za;
	for (int m = 0; m < n; m++) {
		e[m] = za;
		e[n + m] = zg;
		za = make_double2(za.x * ca - za.y * sa, za.x * sa + za.y * ca);
		zg = make_double2(zg.x * cg - zg.y * sg, zg.x * sg + zg.y * cg);
	}
	cudaStream_t st = r->leg->comp_stream;
	cudaMemcpyAsync(r->d_e, e.data(), sizeof(double2) * 2 * n, cudaMemcpyHostToDevice, st);
	launch_plm_table(r->leg, cb, sb, r->d_plm, st);
	r->ready = shtb_cuda_ok(cudaStreamSynchronize(st), "rotation angles") ? 1 : 0;
}

extern "C" void shtns_rotation_set_angles_ZXZ(shtns_rot r, double alpha, double beta, double gamma)
{
	shtns_rotation_set_angles_ZYZ(r, alpha + M_PI / 2, beta, gamma - M_PI / 2);
}

extern "C" void shtns_rotation_set_angle_axis(shtns_rot r, double theta, double Vx, double Vy, double Vz)
{
	if (!r) return;
	if (Vx == 0 && Vy == 0) {         // about z
		if (Vz < 0) theta = -theta;
		shtns_rotation_set_angles_ZYZ(r, theta, 0, 0);
		return;
	}
	// unit quaternion (c, V sin(theta/2) / |V|) -> Euler angles (extrinsic ZYZ, swapped to intrinsic)
	const double s = std::sin(0.5 * theta), c = std::cos(0.5 * theta);
	const double nrm = s / std::sqrt(Vx * Vx + Vy * Vy + Vz * Vz);
	Vx *= nrm; Vy *= nrm; Vz *= nrm;
	const double beta = std::acos(1.0 - 2.0 * (Vx * Vx + Vy * Vy));
	const double alpha = std::atan2(Vy * Vz - c * Vx, c * Vy + Vx * Vz);
	const double gamma = std::atan2(Vy * Vz + c * Vx, c * Vy - Vx * Vz);
	shtns_rotation_set_angles_ZYZ(r, gamma, beta, alpha);
}

extern "C" int shtns_rotation_wigner_d_matrix(shtns_rot r, const int l, double* mx)
{
	if (!r || !mx || l < 0 || l > r->lmax) { shtb_set_error(1, "wigner_d_matrix: 0 <= l <= lmax not satisfied"); return 0; }
	if (!r->ready) { shtb_set_error(1, "wigner_d_matrix: angles not set"); return 0; }
	if (l == 0) { mx[0] = 1.0; return 1; }
	const long w = 2 * l + 1;
	if (!rot_buf(r, sizeof(double) * w * w)) return 0;
	RotParams p = rot_params(r);
	p.wig = static_cast<double*>(r->d_buf);
	p.l0 = l; p.l1 = l;
	cudaStream_t st = r->leg->comp_stream;
	const int nt = std::min(ROT_NT, (l + 1 + 31) / 32 * 32);
	const int kc = (l + 1 + nt - 1) / nt;
	const size_t smem = sizeof(double) * (4 * (size_t)(l + 2) + 256);
	if (kc <= 1) launch_rot<1>(p, nt, smem, st);
	else if (kc <= 2) launch_rot<2>(p, nt, smem, st);
	else if (kc <= 4) launch_rot<4>(p, nt, smem, st);
	else launch_rot<8>(p, nt, smem, st);
	shtb_count_launch();
	if (!shtb_cuda_ok(cudaGetLastError(), "Wigner matrix launch")) return 0;
	cudaMemcpyAsync(mx, p.wig, sizeof(double) * w * w, cudaMemcpyDeviceToHost, st);
	if (!shtb_cuda_ok(cudaStreamSynchronize(st), "Wigner matrix")) return 0;
	return (int) w;
}

extern "C" void shtns_rotation_apply_real(shtns_rot r, cplx* Qlm, cplx* Rlm) { rot_apply(r, Qlm, Rlm, 0); }
extern "C" void shtns_rotation_apply_cplx(shtns_rot r, cplx* Zlm, cplx* Rlm) { rot_apply(r, Zlm, Rlm, 1); }

// ---- rotations through a plan (sht_func.c:37-53, 337-385) ----
extern "C" void SH_Zrotate(shtns_cfg s, cplx* Qlm, double alpha, cplx* Rlm)
{
	if (!s || !Qlm || !Rlm) { shtb_set_error(1, "SH_Zrotate: null argument"); return; }
	const long n = s->nlm;
	void* d = nullptr;
	if (!shtb_cuda_ok(cudaMalloc(&d, 2 * sizeof(double2) * n), "SH_Zrotate buffers")) return;
	double2* q = static_cast<double2*>(d);
	cudaStream_t st = s->comp_stream;
	cudaMemcpyAsync(q, Qlm, sizeof(double2) * n, cudaMemcpyHostToDevice, st);
	dim3 grid((s->lmax + 1 + 127) / 128, s->mmax + 1);
	zrotate_kernel<<<grid, 128, 0, st>>>(q, q + n, s->lmax, s->mmax, s->mres, alpha);
	shtb_count_launch();
	if (shtb_cuda_ok(cudaGetLastError(), "SH_Zrotate launch"))
		cudaMemcpyAsync(Rlm, q + n, sizeof(double2) * n, cudaMemcpyDeviceToHost, st);
	shtb_cuda_ok(cudaStreamSynchronize(st), "SH_Zrotate");
	cudaFree(d);
}

// Rotations about the y and x axes through a plan (mres = 1, mmax = lmax, as
// the reference requires): the same active rotation as shtns_rotation_* with
// ZYZ angles (0, alpha, 0) about y, and the angle-axis form about x.
static void plan_rotation(shtns_cfg s, cplx* Qlm, cplx* Rlm, int axis, double angle)
{
	if (!s || !Qlm || !Rlm) { shtb_set_error(1, "rotation: null argument"); return; }
	if (s->mres != 1 || s->mmax < s->lmax) { shtb_set_error(1, "truncature makes rotation not closed."); return; }
	shtns_rot r = shtns_rotation_create(s->lmax, s->mmax, s->norm_flags);
	if (!r) return;
	cushtns_set_streams(r->leg, s->comp_stream, nullptr);
	if (axis == 1) shtns_rotation_set_angles_ZYZ(r, 0.0, angle, 0.0);
	else shtns_rotation_set_angle_axis(r, angle, 1.0, 0.0, 0.0);
	shtns_rotation_apply_real(r, Qlm, Rlm);
	shtns_rotation_destroy(r);
}

extern "C" void SH_Yrotate(shtns_cfg s, cplx* Qlm, double alpha, cplx* Rlm) { plan_rotation(s, Qlm, Rlm, 1, alpha); }
extern "C" void SH_Yrotate90(shtns_cfg s, cplx* Qlm, cplx* Rlm) { plan_rotation(s, Qlm, Rlm, 1, M_PI / 2); }
extern "C" void SH_Xrotate90(shtns_cfg s, cplx* Qlm, cplx* Rlm) { plan_rotation(s, Qlm, Rlm, 0, M_PI / 2); }
