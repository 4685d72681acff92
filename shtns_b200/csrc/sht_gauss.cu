// Gauss-Legendre nodes and weights on the GPU, one thread per north node.
//
// Algorithm (the reference's gauss_nodes, sht_legendre.c:763-811, and the
// textbook Newton iteration of Numerical Recipes' gauleg): start from the
// asymptotic guess x ~ (1 - (n-1)/(8 n^3)) cos(pi (4i+3)/(4n+2)), evaluate
// P_n and P_{n-1} by the three-term recurrence l P_l = (2l-1) x P_{l-1} -
// (l-1) P_{l-2}, and take Newton steps x -= P_n (1-x^2) / (n (P_{n-1} - x P_n)).
// The weight is w = 2 (1-x^2) / (n (P_{n-1} - x P_n))^2.
//
// Precision: a few Newton steps in FP64 bring x to within a few units in the
// last place; two more steps with the recurrence in double-double arithmetic
// (pairs hi + lo, about 106 bits) make the node and weight correct to well
// below half an FP64 ulp before they are rounded, which is what the
// reference gets from long double (64-bit mantissa).  sin(theta) is the
// double-double sqrt((1-x)(1+x)) of the node as rounded to FP64, so every
// table of the plan describes the same point.
//
// Double-double operations are the error-free transforms of Knuth (TwoSum)
// and Dekker (Fast2Sum), with the product error from one FMA, composed as in
// Hida, Li & Bailey, "Algorithms for quad-double precision floating point
// arithmetic" (ARITH-15, 2001).
#include "sht_internal.h"

namespace {

struct dd { double hi, lo; };

__device__ __forceinline__ dd two_sum(double a, double b)
{
	const double s = a + b;
	const double bb = s - a;
	return {s, (a - (s - bb)) + (b - bb)};
}

__device__ __forceinline__ dd fast_two_sum(double a, double b)   // |a| >= |b|
{
	const double s = a + b;
	return {s, b - (s - a)};
}

__device__ __forceinline__ dd two_prod(double a, double b)
{
	const double p = a * b;
	return {p, fma(a, b, -p)};
}

__device__ __forceinline__ dd dd_add(dd a, dd b)
{
	dd s = two_sum(a.hi, b.hi);
	const dd t = two_sum(a.lo, b.lo);
	s.lo += t.hi;
	s = fast_two_sum(s.hi, s.lo);
	s.lo += t.lo;
	return fast_two_sum(s.hi, s.lo);
}

__device__ __forceinline__ dd dd_neg(dd a) { return {-a.hi, -a.lo}; }

__device__ __forceinline__ dd dd_mul(dd a, dd b)
{
	dd p = two_prod(a.hi, b.hi);
	p.lo = fma(a.hi, b.lo, fma(a.lo, b.hi, p.lo));
	return fast_two_sum(p.hi, p.lo);
}

__device__ __forceinline__ dd dd_mul_d(dd a, double b)
{
	dd p = two_prod(a.hi, b);
	p.lo = fma(a.lo, b, p.lo);
	return fast_two_sum(p.hi, p.lo);
}

// a / b: a long division with three FP64 quotient digits
__device__ __forceinline__ dd dd_div(dd a, dd b)
{
	const double q1 = a.hi / b.hi;
	dd r = dd_add(a, dd_neg(dd_mul_d(b, q1)));
	const double q2 = r.hi / b.hi;
	r = dd_add(r, dd_neg(dd_mul_d(b, q2)));
	const double q3 = r.hi / b.hi;
	return dd_add(fast_two_sum(q1, q2), dd{q3, 0.0});
}

// (l-1)/l for an integer l >= 1: the FP64 quotient and its exact remainder
__device__ __forceinline__ dd ratio_lm1_l(long l)
{
	const double a = (double)(l - 1), b = (double) l;
	const double q = a / b;
	return {q, fma(-q, b, a) / b};
}

// P_n and P_{n-1} at x, FP64.  l P_l = l x P_{l-1} + (l-1) (x P_{l-1} - P_{l-2}).
__device__ void legendre_pair_d(int n, double x, double& pn, double& pn1)
{
	double p1 = x, p2 = 1.0;
	for (long l = 2; l <= n; l++) {
		const double xp = x * p1;
		const double p = fma((double)(l - 1) / (double) l, xp - p2, xp);
		p2 = p1; p1 = p;
	}
	pn = p1; pn1 = p2;
}

// the same in double-double
__device__ void legendre_pair_dd(int n, dd x, dd& pn, dd& pn1)
{
	dd p1 = x, p2 = {1.0, 0.0};
	for (long l = 2; l <= n; l++) {
		const dd xp = dd_mul(x, p1);
		const dd p = dd_add(xp, dd_mul(ratio_lm1_l(l), dd_add(xp, dd_neg(p2))));
		p2 = p1; p1 = p;
	}
	pn = p1; pn1 = p2;
}

__global__ void gauss_nodes_kernel(int n, double* __restrict__ xo, double* __restrict__ so, double* __restrict__ wo)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n / 2) return;
	const double pi = 3.141592653589793238462643383279502884;
	double z = (1.0 - (n - 1.0) / (8.0 * n * n * (double) n)) * cos(pi * (4.0 * i + 3.0) / (4.0 * n + 2.0));
	// FP64 Newton steps (at most 10, as the reference)
	for (int it = 0; it < 10; it++) {
		double pn, pn1;
		legendre_pair_d(n, z, pn, pn1);
		const double pp = n * (pn1 - z * pn);
		const double dz = pn * (1.0 - z * z) / pp;
		z -= dz;
		if (fabs(dz) <= fabs(z) * 2.3e-16) break;
	}
	// two double-double Newton steps from the FP64 node
	dd x = {z, 0.0};
	dd pn, pn1, pp;
	const dd one = {1.0, 0.0};
	for (int it = 0; it < 2; it++) {
		legendre_pair_dd(n, x, pn, pn1);
		pp = dd_mul_d(dd_add(pn1, dd_neg(dd_mul(x, pn))), (double) n);
		const dd s2 = dd_add(one, dd_neg(dd_mul(x, x)));
		x = dd_add(x, dd_neg(dd_div(dd_mul(pn, s2), pp)));
	}
	legendre_pair_dd(n, x, pn, pn1);
	pp = dd_mul_d(dd_add(pn1, dd_neg(dd_mul(x, pn))), (double) n);
	const dd s2 = dd_add(one, dd_neg(dd_mul(x, x)));
	const dd w = dd_div(dd_mul_d(s2, 2.0), dd_mul(pp, pp));
	const double xr = x.hi + x.lo;                 // node rounded to FP64
	// sin(theta) of the rounded node: sqrt((1 - xr)(1 + xr)) in double-double
	const dd a = dd_mul(two_sum(1.0, -xr), two_sum(1.0, xr));
	const double s0 = sqrt(a.hi);
	const dd e = dd_add(a, dd_neg(two_prod(s0, s0)));
	xo[i] = xr;
	so[i] = s0 + e.hi / (2.0 * s0);
	wo[i] = w.hi + w.lo;
}

} // namespace

// Nodes x (decreasing, north half), sin(theta) and weights of the n-point
// Gauss-Legendre rule on the current device.  Returns false (error recorded)
// if the GPU work fails.
bool gauss_grid_gpu(int n, std::vector<double>& x, std::vector<double>& st, std::vector<double>& w)
{
	const int m = n / 2;
	x.assign(m, 0.0); st.assign(m, 0.0); w.assign(m, 0.0);
	if (m == 0) return true;
	double* d = nullptr;
	if (!shtb_cuda_ok(cudaMalloc(&d, sizeof(double) * 3 * (size_t) m), "Gauss nodes")) return false;
	gauss_nodes_kernel<<<(m + 127) / 128, 128>>>(n, d, d + m, d + 2 * m);
	shtb_count_launch();
	bool ok = shtb_cuda_ok(cudaGetLastError(), "Gauss nodes kernel");
	ok = ok && shtb_cuda_ok(cudaMemcpy(x.data(), d, sizeof(double) * m, cudaMemcpyDeviceToHost), "Gauss nodes");
	ok = ok && shtb_cuda_ok(cudaMemcpy(st.data(), d + m, sizeof(double) * m, cudaMemcpyDeviceToHost), "Gauss nodes");
	ok = ok && shtb_cuda_ok(cudaMemcpy(w.data(), d + 2 * m, sizeof(double) * m, cudaMemcpyDeviceToHost), "Gauss nodes");
	cudaFree(d);
	if (!ok) return false;
	for (int i = 1; i < m; i++)
		if (!(x[i] < x[i - 1])) { shtb_set_error(2, "bad gauss points"); return false; }
	return true;
}
