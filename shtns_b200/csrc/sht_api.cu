// Transform entry points of shtns_b200.
//
// Device-pointer transforms (cu_*, reference sht_gpu.cu:495-577) enqueue three
// kernels per direction on the plan's compute stream and return:
//   synthesis: coefficient prologue -> Legendre contraction -> phi FFT
//   analysis:  phi FFT -> Legendre contraction -> coefficient epilogue
// Host-pointer transforms (SH_to_spat, ..., reference sht_com.c:26-126 with the
// GPU offload of sht_gpu.cu:584-1489) copy their inputs to plan-owned device
// staging, run the same pipeline and copy the outputs back before returning.
#include "sht_internal.h"

#include <cstring>
#include <cstdint>
#include <cstdlib>
#include <algorithm>

namespace {

bool ensure(void** p, size_t* cap, size_t bytes, const char* what)
{
	if (*cap >= bytes && *p) return true;
	if (*p) cudaFree(*p);
	*p = nullptr; *cap = 0;
	if (cudaMalloc(p, bytes) != cudaSuccess) {
		cudaGetLastError();
		shtb_set_error(3, std::string("out of device memory for ") + what);
		return false;
	}
	*cap = bytes;
	return true;
}

} // namespace

// bufs: 1 = coefficient buffer, 2 = Fourier buffer (0: shape only, nothing allocated)
bool setup_job(shtns_cfg s, Job& j, int ncomp, const int* types, int ltr, unsigned bufs)
{
	if (!s || !s->grid_set) { shtb_set_error(1, "transform on a plan without grid"); return false; }
	if (ltr < 0) { shtb_set_error(1, "negative truncation degree"); return false; }
	j.ncomp = ncomp;
	for (int c = 0; c < 3; c++) j.type[c] = (c < ncomp) ? types[c] : 0;
	j.nf = s->batch;
	j.nfc = j.nf * ncomp;
	j.ncol = 16 * ((j.nfc + 3) / 4);
	j.llim = std::min<int>(ltr, s->lmax);
	j.mlim = std::min<int>(s->mmax, j.llim / s->mres);
	j.vec_extra = 0;
	for (int c = 0; c < ncomp; c++) if (types[c]) j.vec_extra = 1;
	// work buffers
	size_t qq_bytes = sizeof(double) * (size_t) s->ktot * j.ncol;
	size_t F_bytes = sizeof(double2) * (size_t) j.nfc * (s->mmax + 1) * s->nlat;
	size_t cq = s->qq_cap * sizeof(double), cf = s->F_cap * sizeof(double2);
	if (bufs & 1) {
		if (!ensure((void**) &s->d_qq, &cq, qq_bytes, "coefficient buffer")) { s->qq_cap = 0; return false; }
		s->qq_cap = cq / sizeof(double);
	}
	if (bufs & 2) {
		if (!ensure((void**) &s->d_F, &cf, F_bytes, "Fourier buffer")) { s->F_cap = 0; return false; }
		s->F_cap = cf / sizeof(double2);
	}
	return true;
}

LegParams leg_params(shtns_cfg s, const Job& j)
{
	LegParams p;
	memset(&p, 0, sizeof(p));
	p.nlat = s->nlat; p.nlat_2 = s->nlat_2; p.llim = j.llim; p.mlim = j.mlim; p.mres = s->mres;
	p.vec_extra = j.vec_extra; p.ncol = j.ncol; p.nfc = j.nfc;
	p.south_first = s->south_first; p.robert = s->robert;
	p.mpos_inv = 1.0 / s->mpos_renorm;
	p.nphi = (double) s->nphi;
	p.x = s->d_x; p.x2 = s->d_x2; p.sinv = s->d_sinv; p.w = s->d_w; p.c = s->d_c;
	p.ck = s->d_ck; p.mt = s->mt; p.ckseg = s->ckseg; p.tile_wm = s->tile_wm;
	p.nf = j.nf;
	for (int c = 0; c < 3; c++) p.ctype[c] = j.type[c];
	p.qq = s->d_qq; p.F = s->d_F;
	p.fstride = (long)(s->mmax + 1) * s->nlat;
	return p;
}

PrepParams prep_params(shtns_cfg s, const Job& j)
{
	PrepParams p;
	memset(&p, 0, sizeof(p));
	p.lmax = s->lmax; p.llim = j.llim; p.mlim = j.mlim; p.mres = s->mres;
	p.nf = j.nf; p.ncomp = j.ncomp; p.ncol = j.ncol;
	for (int c = 0; c < 3; c++) p.comp_type[c] = j.type[c];
	p.spec_dist = s->spec_dist;
	p.xs = s->d_xs; p.xa = s->d_xa;
	p.stdt_lo = s->d_stdt_lo; p.stdt_hi = s->d_stdt_hi; p.van_lo = s->d_van_lo; p.van_hi = s->d_van_hi;
	p.l2 = s->d_l2; p.mt = s->mt; p.qq = s->d_qq;
	return p;
}

// nrows: grid rows transformed (the plan's nlat, or a block of them)
FftParams fft_params(shtns_cfg s, const Job& j, int nrows)
{
	if (nrows <= 0) nrows = s->nlat;
	FftParams p;
	memset(&p, 0, sizeof(p));
	p.N = s->nphi; p.nlat = s->nlat; p.mlim = j.mlim;
	p.nradix = (int) s->fft_radix.size();
	p.rcode = 0;
	int rmin = 8;
	for (int i = 0; i < p.nradix; i++) {
		p.rcode |= (unsigned long long) s->fft_radix[i] << (4 * i);
		rmin = std::min(rmin, s->fft_radix[i]);
	}
	(void) rmin;
	// latitude pairs per CTA: the largest of 4, 2, 1 whose two shared-memory
	// buffers fit in about 110 KB (two CTAs per SM); SHTNS_B200_FFT_PAIRS
	// overrides (tuning knob, clamped to what fits in 227 KB).
	int S = 4;
	while (S > 1 && fft_smem_bytes(s->nphi, S) > 112 * 1024) S /= 2;
	int want = s->fft_pairs;
	if (const char* e = getenv("SHTNS_B200_FFT_PAIRS")) want = atoi(e);
	if (want == 1 || want == 2 || want == 4 || want == 8) {
		// fused chains keep one buffer, the generic kernels two
		const bool fused = fft_fused_available(s->nphi) && s->fft_generic != 1;
		S = want;
		while (S > 1 && fft_smem_bytes(s->nphi, S) / (fused ? 2 : 1) > 227 * 1024) S /= 2;
		if (!fused && S > 4) S = 4;
	}
	while (S > 1 && 2 * S > nrows) S /= 2;
	p.S = S;
	p.tw = s->d_tw; p.F = s->d_F;
	p.fstride = (long)(s->mmax + 1) * s->nlat;
	p.nf = j.nf; p.spat_dist = s->spat_dist;
	p.phi_contiguous = s->phi_contiguous;
	// generic kernels need two buffers
	p.generic = (s->fft_generic == 1) ? (fft_smem_bytes(s->nphi, 1) <= 227 * 1024 ? 1 : 0) : s->fft_generic;
	p.extra_tx = s->fft_extra_tx;
	p.tw1 = s->d_tw4;
	p.tw2 = s->d_tw4 ? s->d_tw4 + 96 : nullptr;
	p.scratch = nullptr;
	return p;
}

namespace {

int aligned16(const void* a, const void* b, const void* c, long dist)
{
	auto ok = [](const void* x) { return ((uintptr_t) x & 15) == 0; };
	return ok(a) && ok(b) && ok(c) && (dist % 2 == 0);
}

bool check_launch(const char* what)
{
	return shtb_cuda_ok(cudaGetLastError(), what);
}

// ---- device pipelines ----
// adjoint = 1 runs the transpose of the analysis (ncomp must be 1): the
// analysis Ishioka basis in the prologue and the quadrature weights applied
// to the rows in the Legendre epilogue.
void run_synth(shtns_cfg s, int ncomp, const int* types, const cplx* Q, const cplx* S, const cplx* T,
               double* o0, double* o1, double* o2, int ltr, int adjoint = 0)
{
	Job j;
	if (!setup_job(s, j, ncomp, types, ltr)) return;
	PrepParams pp = prep_params(s, j);
	if (adjoint) pp.xs = s->d_xa;
	pp.Q = reinterpret_cast<const double2*>(Q);
	pp.S = reinterpret_cast<const double2*>(S);
	pp.T = reinterpret_cast<const double2*>(T);
	shtb_stage_begin(s, 0);
	launch_prep_synth(pp, s->comp_stream);
	shtb_stage_end(s);
	LegParams lp = leg_params(s, j);
	lp.adjoint = adjoint;
	shtb_stage_begin(s, 1);
	if (s->split_ns) launch_leg_synth_split(s, lp, s->comp_stream);
	else if (!launch_ftab_synth(s, lp, s->comp_stream)) launch_leg_synth(lp, s->comp_stream);
	shtb_stage_end(s);
	FftParams fp = fft_params(s, j);
	fp.spat[0] = o0; fp.spat[1] = o1; fp.spat[2] = o2;
	fp.vec2 = aligned16(o0, o1, o2, s->spat_dist);
	shtb_stage_begin(s, 2);
	launch_fft_synth(fp, j.nfc, s->comp_stream);
	shtb_stage_end(s);
	check_launch("synthesis launch");
}

// adjoint = 1 runs the transpose of the synthesis (ncomp must be 1): no
// quadrature weights, the factor nphi (2 - delta_m0) and the synthesis
// Ishioka basis in the epilogue.
void run_analys(shtns_cfg s, int ncomp, const int* types, const double* i0, const double* i1, const double* i2,
                cplx* Qo, cplx* So, cplx* To, int ltr, int adjoint = 0)
{
	Job j;
	if (!setup_job(s, j, ncomp, types, ltr)) return;
	FftParams fp = fft_params(s, j);
	fp.spat_in[0] = i0; fp.spat_in[1] = i1; fp.spat_in[2] = i2;
	fp.vec2 = aligned16(i0, i1, i2, s->spat_dist);
	if (s->d_tw4 && !s->phi_contiguous && fp.vec2 && s->fft_generic == 0) {
		// the four-step FFT analysis of nphi = 12288 needs a grid per field-component of scratch
		// (without room for it the direct kernels run instead)
		const size_t b = sizeof(double) * (size_t) j.nfc * s->nphi * s->nlat;
		if (s->fscr_cap < b) {
			if (s->d_fscr) cudaFree(s->d_fscr);
			s->d_fscr = nullptr; s->fscr_cap = 0;
			if (cudaMalloc(reinterpret_cast<void**>(&s->d_fscr), b) == cudaSuccess) s->fscr_cap = b;
			else { cudaGetLastError(); s->d_fscr = nullptr; }
		}
		fp.scratch = s->d_fscr;
	}
	shtb_stage_begin(s, 3);
	launch_fft_analys(fp, j.nfc, s->comp_stream);
	shtb_stage_end(s);
	LegParams lp = leg_params(s, j);
	lp.adjoint = adjoint;
	int kmax_all = 0;
	for (int im = 0; im <= j.mlim; im++) kmax_all = std::max(kmax_all, (j.llim + j.vec_extra - im * s->mres) / 2 + 1);
	shtb_stage_begin(s, 4);
	if (s->split_ns && s->split_form == 0) launch_ptab_analys(s, lp, s->comp_stream);
	else launch_leg_analys(lp, kmax_all, s->comp_stream);
	shtb_stage_end(s);
	PrepParams pp = prep_params(s, j);
	if (adjoint) pp.xa = s->d_xs;
	pp.Qo = reinterpret_cast<double2*>(Qo);
	pp.So = reinterpret_cast<double2*>(So);
	pp.To = reinterpret_cast<double2*>(To);
	shtb_stage_begin(s, 5);
	launch_post_analys_m(pp, s->mmax, s->comp_stream);
	shtb_stage_end(s);
	check_launch("analysis launch");
}

const int T_SCAL[1] = {0};
const int T_VEC[2] = {1, 2};
const int T_QST[3] = {0, 1, 2};

// ---- host-pointer forms: stage through device memory ----
struct Stage {
	double2* spec[3];
	double* spat[3];
};

bool stage_alloc(shtns_cfg s, int nspec, int nspatial, Stage& st)
{
	const size_t spec_elems = (size_t)(s->batch - 1) * s->spec_dist + s->nlm;
	const size_t spat_elems = (size_t)(s->batch - 1) * s->spat_dist + s->nspat;
	const size_t spec_b = (sizeof(double2) * spec_elems + 255) & ~(size_t) 255;
	const size_t spat_b = (sizeof(double) * spat_elems + 255) & ~(size_t) 255;
	const size_t total = nspec * spec_b + nspatial * spat_b;
	if (!ensure(&s->d_stage, &s->stage_cap, total, "staging buffers")) return false;
	char* base = (char*) s->d_stage;
	for (int i = 0; i < 3; i++) { st.spec[i] = nullptr; st.spat[i] = nullptr; }
	for (int i = 0; i < nspec; i++) { st.spec[i] = (double2*) base; base += spec_b; }
	for (int i = 0; i < nspatial; i++) { st.spat[i] = (double*) base; base += spat_b; }
	return true;
}


// Host-pointer transforms, pipelined over chunks of fields (up to 8 chunks):
// host->device copies of chunk c+1 on the transfer stream and device->host
// copies of chunk c on a second copy stream overlap the transforms of chunk c
// (c+1) on the compute stream; events order each chunk's copies and
// transforms.  Page-locked host arrays (shtns_malloc, cudaHostAlloc,
// cudaHostRegister) are copied fully asynchronously, both directions at once;
// pageable arrays go through the driver's staging, and the next chunk's
// transforms are enqueued before a chunk's device->host copy (which returns
// only when done), so the GPU keeps working while the host copies.
// (The reference offloads sht_gpu.cu:584-1489 overlap per-component copies
// with the transforms of the next component in the same way.)
struct HostChunks {
	int B, fpc, nch;
};

HostChunks host_chunks(shtns_cfg s)
{
	HostChunks h;
	h.B = s->batch;
	const int want = std::min(h.B, 8);
	h.fpc = (h.B + want - 1) / want;
	h.nch = (h.B + h.fpc - 1) / h.fpc;
	return h;
}

bool copy_resources(shtns_cfg s, int nev)
{
	if (!s->d2h_stream && cudaStreamCreateWithFlags(&s->d2h_stream, cudaStreamNonBlocking) != cudaSuccess) {
		cudaGetLastError();
		s->d2h_stream = nullptr;
		shtb_set_error(2, "could not create the copy stream");
		return false;
	}
	if (!s->xfer_stream) {
		if (cudaStreamCreateWithFlags(&s->xfer_stream, cudaStreamNonBlocking) != cudaSuccess) {
			cudaGetLastError();
			shtb_set_error(2, "could not create the transfer stream");
			return false;
		}
		s->own_xfer = 1;
	}
	while ((int) s->xev.size() < nev) {
		cudaEvent_t e;
		if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
			cudaGetLastError();
			shtb_set_error(2, "could not create copy events");
			return false;
		}
		s->xev.push_back(e);
	}
	return true;
}

void h_synth(shtns_cfg s, int ncomp, const int* types, const cplx* Q, const cplx* S, const cplx* T,
             double* o0, double* o1, double* o2, int ltr)
{
	if (!s || !s->grid_set) { shtb_set_error(1, "transform on a plan without grid"); return; }
	const int nin = (Q ? 1 : 0) + (S ? 1 : 0) + (T ? 1 : 0);
	Stage st;
	if (!stage_alloc(s, nin, ncomp, st)) return;
	const HostChunks h = host_chunks(s);
	if (!copy_resources(s, 2 * h.nch)) return;
	cudaStream_t cs = s->comp_stream, xh = s->xfer_stream, xd = s->d2h_stream;
	const cplx* hin[3] = {Q, S, T};
	double* hout[3] = {o0, o1, o2};
	double2* din[3] = {nullptr, nullptr, nullptr};
	{
		int k = 0;
		for (int i = 0; i < 3; i++) if (hin[i]) din[i] = st.spec[k++];
	}
	const long sd = s->spec_dist, pd = s->spat_dist;
	auto h2d = [&](int c) {
		const int f0 = c * h.fpc, nf = std::min(h.fpc, h.B - f0);
		const size_t b = sizeof(double2) * ((size_t)(nf - 1) * sd + s->nlm);
		for (int i = 0; i < 3; i++)
			if (hin[i]) cudaMemcpyAsync(din[i] + f0 * sd, reinterpret_cast<const double2*>(hin[i]) + f0 * sd, b,
			                            cudaMemcpyHostToDevice, xh);
		cudaEventRecord(s->xev[2 * c], xh);
	};
	auto compute = [&](int c) {
		const int f0 = c * h.fpc, nf = std::min(h.fpc, h.B - f0);
		cudaStreamWaitEvent(cs, s->xev[2 * c], 0);
		s->batch = nf;
		auto in = [&](int i) { return din[i] ? reinterpret_cast<const cplx*>(din[i] + f0 * sd) : (const cplx*) nullptr; };
		run_synth(s, ncomp, types, in(0), in(1), in(2), st.spat[0] ? st.spat[0] + f0 * pd : nullptr,
		          st.spat[1] ? st.spat[1] + f0 * pd : nullptr, st.spat[2] ? st.spat[2] + f0 * pd : nullptr, ltr);
		s->batch = h.B;
		cudaEventRecord(s->xev[2 * c + 1], cs);
	};
	auto d2h = [&](int c) {
		const int f0 = c * h.fpc, nf = std::min(h.fpc, h.B - f0);
		const size_t b = sizeof(double) * ((size_t)(nf - 1) * pd + s->nspat);
		cudaStreamWaitEvent(xd, s->xev[2 * c + 1], 0);
		for (int i = 0; i < ncomp; i++) cudaMemcpyAsync(hout[i] + f0 * pd, st.spat[i] + f0 * pd, b, cudaMemcpyDeviceToHost, xd);
	};
	h2d(0);
	compute(0);
	for (int c = 0; c < h.nch; c++) {
		if (c + 1 < h.nch) { h2d(c + 1); compute(c + 1); }
		d2h(c);
	}
	shtb_cuda_ok(cudaStreamSynchronize(xd), "synthesis");
}

void h_analys(shtns_cfg s, int ncomp, const int* types, const double* i0, const double* i1, const double* i2,
              cplx* Qo, cplx* So, cplx* To, int ltr)
{
	if (!s || !s->grid_set) { shtb_set_error(1, "transform on a plan without grid"); return; }
	Stage st;
	if (!stage_alloc(s, ncomp, ncomp, st)) return;
	const HostChunks h = host_chunks(s);
	if (!copy_resources(s, 2 * h.nch)) return;
	cudaStream_t cs = s->comp_stream, xh = s->xfer_stream, xd = s->d2h_stream;
	const double* hin[3] = {i0, i1, i2};
	cplx* hout[3] = {Qo, So, To};
	double2* dout[3] = {nullptr, nullptr, nullptr};
	{
		int k = 0;
		for (int i = 0; i < 3; i++) if (hout[i]) dout[i] = st.spec[k++];
	}
	const long sd = s->spec_dist, pd = s->spat_dist;
	auto h2d = [&](int c) {
		const int f0 = c * h.fpc, nf = std::min(h.fpc, h.B - f0);
		const size_t b = sizeof(double) * ((size_t)(nf - 1) * pd + s->nspat);
		for (int i = 0; i < ncomp; i++) cudaMemcpyAsync(st.spat[i] + f0 * pd, hin[i] + f0 * pd, b, cudaMemcpyHostToDevice, xh);
		cudaEventRecord(s->xev[2 * c], xh);
	};
	auto compute = [&](int c) {
		const int f0 = c * h.fpc, nf = std::min(h.fpc, h.B - f0);
		cudaStreamWaitEvent(cs, s->xev[2 * c], 0);
		s->batch = nf;
		auto out = [&](int i) { return dout[i] ? reinterpret_cast<cplx*>(dout[i] + f0 * sd) : (cplx*) nullptr; };
		run_analys(s, ncomp, types, st.spat[0] + f0 * pd, st.spat[1] ? st.spat[1] + f0 * pd : nullptr,
		           st.spat[2] ? st.spat[2] + f0 * pd : nullptr, out(0), out(1), out(2), ltr);
		s->batch = h.B;
		cudaEventRecord(s->xev[2 * c + 1], cs);
	};
	auto d2h = [&](int c) {
		const int f0 = c * h.fpc, nf = std::min(h.fpc, h.B - f0);
		const size_t b = sizeof(double2) * ((size_t)(nf - 1) * sd + s->nlm);
		cudaStreamWaitEvent(xd, s->xev[2 * c + 1], 0);
		for (int i = 0; i < 3; i++)
			if (hout[i]) cudaMemcpyAsync(reinterpret_cast<double2*>(hout[i]) + f0 * sd, dout[i] + f0 * sd, b,
			                             cudaMemcpyDeviceToHost, xd);
	};
	h2d(0);
	compute(0);
	for (int c = 0; c < h.nch; c++) {
		if (c + 1 < h.nch) { h2d(c + 1); compute(c + 1); }
		d2h(c);
	}
	shtb_cuda_ok(cudaStreamSynchronize(xd), "analysis");
}

} // namespace

// ---------------------------------------------------------------------------
extern "C" int shtns_set_batch(shtns_cfg s, int howmany, long spec_dist, long spat_dist)
{
	if (!s || howmany < 1) { shtb_set_error(1, "shtns_set_batch: invalid arguments"); return -1; }
	if (spec_dist < (long) s->nlm) spec_dist = s->nlm;
	if (spat_dist < (long) s->nspat) spat_dist = s->nspat;
	s->batch = howmany; s->spec_dist = spec_dist; s->spat_dist = spat_dist;
	return 0;
}

// ---- device-pointer API (shtns_cuda.h) ----
extern "C" void cu_SH_to_spat(shtns_cfg s, cplx* Qlm, double* Vr, int ltr)
{ run_synth(s, 1, T_SCAL, Qlm, nullptr, nullptr, Vr, nullptr, nullptr, ltr); }

extern "C" void cu_spat_to_SH(shtns_cfg s, double* Vr, cplx* Qlm, int ltr)
{ run_analys(s, 1, T_SCAL, Vr, nullptr, nullptr, Qlm, nullptr, nullptr, ltr); }

extern "C" void cu_SHsphtor_to_spat(shtns_cfg s, cplx* Slm, cplx* Tlm, double* Vt, double* Vp, int ltr)
{ run_synth(s, 2, T_VEC, nullptr, Slm, Tlm, Vt, Vp, nullptr, ltr); }

extern "C" void cu_spat_to_SHsphtor(shtns_cfg s, double* Vt, double* Vp, cplx* Slm, cplx* Tlm, int ltr)
{ run_analys(s, 2, T_VEC, Vt, Vp, nullptr, nullptr, Slm, Tlm, ltr); }

extern "C" void cu_SHqst_to_spat(shtns_cfg s, cplx* Qlm, cplx* Slm, cplx* Tlm, double* Vr, double* Vt, double* Vp, int ltr)
{ run_synth(s, 3, T_QST, Qlm, Slm, Tlm, Vr, Vt, Vp, ltr); }

extern "C" void cu_spat_to_SHqst(shtns_cfg s, double* Vr, double* Vt, double* Vp, cplx* Qlm, cplx* Slm, cplx* Tlm, int ltr)
{ run_analys(s, 3, T_QST, Vr, Vt, Vp, Qlm, Slm, Tlm, ltr); }

// ---- adjoints (shtns_b200.h) ----
extern "C" void cu_SH_to_spat_adjoint(shtns_cfg s, double* Vg, cplx* Qg, int ltr)
{ run_analys(s, 1, T_SCAL, Vg, nullptr, nullptr, Qg, nullptr, nullptr, ltr, 1); }

extern "C" void cu_spat_to_SH_adjoint(shtns_cfg s, cplx* Qg, double* Vg, int ltr)
{ run_synth(s, 1, T_SCAL, Qg, nullptr, nullptr, Vg, nullptr, nullptr, ltr, 1); }

// Single-precision device transforms (shtns_cuda.h:410,414): FP32 arrays in
// and out, converted to FP64 in the plan's staging buffer, transformed in FP64
// and rounded back to FP32 (the reference computes these in FP32).
namespace {
__global__ void f2d_kernel(const float* __restrict__ in, double* __restrict__ out, long n)
{
	for (long i = blockIdx.x * (long) blockDim.x + threadIdx.x; i < n; i += (long) gridDim.x * blockDim.x) out[i] = in[i];
}
__global__ void d2f_kernel(const double* __restrict__ in, float* __restrict__ out, long n)
{
	for (long i = blockIdx.x * (long) blockDim.x + threadIdx.x; i < n; i += (long) gridDim.x * blockDim.x) out[i] = (float) in[i];
}
void convert(const float* in, double* out, long n, cudaStream_t st)
{
	f2d_kernel<<<(unsigned) std::min<long>((n + 255) / 256, 148 * 16), 256, 0, st>>>(in, out, n);
	shtb_count_launch();
}
void convert(const double* in, float* out, long n, cudaStream_t st)
{
	d2f_kernel<<<(unsigned) std::min<long>((n + 255) / 256, 148 * 16), 256, 0, st>>>(in, out, n);
	shtb_count_launch();
}
} // namespace

extern "C" void cu_SH_to_spat_float(shtns_cfg s, cplx_f* Qlm, float* Vr, int ltr)
{
	if (!s || !s->grid_set) { shtb_set_error(1, "transform on a plan without grid"); return; }
	Stage st;
	if (!stage_alloc(s, 1, 1, st)) return;
	const long nspec = 2 * ((long)(s->batch - 1) * s->spec_dist + s->nlm);
	const long nsp = (long)(s->batch - 1) * s->spat_dist + s->nspat;
	convert(reinterpret_cast<const float*>(Qlm), reinterpret_cast<double*>(st.spec[0]), nspec, s->comp_stream);
	run_synth(s, 1, T_SCAL, reinterpret_cast<cplx*>(st.spec[0]), nullptr, nullptr, st.spat[0], nullptr, nullptr, ltr);
	convert(st.spat[0], Vr, nsp, s->comp_stream);
	shtb_cuda_ok(cudaGetLastError(), "cu_SH_to_spat_float");
}

extern "C" void cu_spat_to_SH_float(shtns_cfg s, float* Vr, cplx_f* Qlm, int ltr)
{
	if (!s || !s->grid_set) { shtb_set_error(1, "transform on a plan without grid"); return; }
	Stage st;
	if (!stage_alloc(s, 1, 1, st)) return;
	const long nspec = 2 * ((long)(s->batch - 1) * s->spec_dist + s->nlm);
	const long nsp = (long)(s->batch - 1) * s->spat_dist + s->nspat;
	convert(Vr, st.spat[0], nsp, s->comp_stream);
	run_analys(s, 1, T_SCAL, st.spat[0], nullptr, nullptr, reinterpret_cast<cplx*>(st.spec[0]), nullptr, nullptr, ltr);
	convert(reinterpret_cast<const double*>(st.spec[0]), reinterpret_cast<float*>(Qlm), nspec, s->comp_stream);
	shtb_cuda_ok(cudaGetLastError(), "cu_spat_to_SH_float");
}

// ---- host-pointer API (shtns.h) ----
extern "C" void SH_to_spat(shtns_cfg s, cplx* Qlm, double* Vr) { h_synth(s, 1, T_SCAL, Qlm, nullptr, nullptr, Vr, nullptr, nullptr, s ? s->lmax : 0); }
extern "C" void SH_to_spat_l(shtns_cfg s, cplx* Qlm, double* Vr, int ltr) { h_synth(s, 1, T_SCAL, Qlm, nullptr, nullptr, Vr, nullptr, nullptr, ltr); }
extern "C" void spat_to_SH(shtns_cfg s, double* Vr, cplx* Qlm) { h_analys(s, 1, T_SCAL, Vr, nullptr, nullptr, Qlm, nullptr, nullptr, s ? s->lmax : 0); }
extern "C" void spat_to_SH_l(shtns_cfg s, double* Vr, cplx* Qlm, int ltr) { h_analys(s, 1, T_SCAL, Vr, nullptr, nullptr, Qlm, nullptr, nullptr, ltr); }

extern "C" void SHsphtor_to_spat(shtns_cfg s, cplx* Slm, cplx* Tlm, double* Vt, double* Vp)
{ h_synth(s, 2, T_VEC, nullptr, Slm, Tlm, Vt, Vp, nullptr, s ? s->lmax : 0); }
extern "C" void SHsphtor_to_spat_l(shtns_cfg s, cplx* Slm, cplx* Tlm, double* Vt, double* Vp, int ltr)
{ h_synth(s, 2, T_VEC, nullptr, Slm, Tlm, Vt, Vp, nullptr, ltr); }
extern "C" void SHsph_to_spat(shtns_cfg s, cplx* Slm, double* Vt, double* Vp)
{ h_synth(s, 2, T_VEC, nullptr, Slm, nullptr, Vt, Vp, nullptr, s ? s->lmax : 0); }
extern "C" void SHsph_to_spat_l(shtns_cfg s, cplx* Slm, double* Vt, double* Vp, int ltr)
{ h_synth(s, 2, T_VEC, nullptr, Slm, nullptr, Vt, Vp, nullptr, ltr); }
extern "C" void SHtor_to_spat(shtns_cfg s, cplx* Tlm, double* Vt, double* Vp)
{ h_synth(s, 2, T_VEC, nullptr, nullptr, Tlm, Vt, Vp, nullptr, s ? s->lmax : 0); }
extern "C" void SHtor_to_spat_l(shtns_cfg s, cplx* Tlm, double* Vt, double* Vp, int ltr)
{ h_synth(s, 2, T_VEC, nullptr, nullptr, Tlm, Vt, Vp, nullptr, ltr); }
extern "C" void spat_to_SHsphtor(shtns_cfg s, double* Vt, double* Vp, cplx* Slm, cplx* Tlm)
{ h_analys(s, 2, T_VEC, Vt, Vp, nullptr, nullptr, Slm, Tlm, s ? s->lmax : 0); }
extern "C" void spat_to_SHsphtor_l(shtns_cfg s, double* Vt, double* Vp, cplx* Slm, cplx* Tlm, int ltr)
{ h_analys(s, 2, T_VEC, Vt, Vp, nullptr, nullptr, Slm, Tlm, ltr); }

extern "C" void SHqst_to_spat(shtns_cfg s, cplx* Qlm, cplx* Slm, cplx* Tlm, double* Vr, double* Vt, double* Vp)
{ h_synth(s, 3, T_QST, Qlm, Slm, Tlm, Vr, Vt, Vp, s ? s->lmax : 0); }
extern "C" void SHqst_to_spat_l(shtns_cfg s, cplx* Qlm, cplx* Slm, cplx* Tlm, double* Vr, double* Vt, double* Vp, int ltr)
{ h_synth(s, 3, T_QST, Qlm, Slm, Tlm, Vr, Vt, Vp, ltr); }
extern "C" void spat_to_SHqst(shtns_cfg s, double* Vr, double* Vt, double* Vp, cplx* Qlm, cplx* Slm, cplx* Tlm)
{ h_analys(s, 3, T_QST, Vr, Vt, Vp, Qlm, Slm, Tlm, s ? s->lmax : 0); }
extern "C" void spat_to_SHqst_l(shtns_cfg s, double* Vr, double* Vt, double* Vp, cplx* Qlm, cplx* Slm, cplx* Tlm, int ltr)
{ h_analys(s, 3, T_QST, Vr, Vt, Vp, Qlm, Slm, Tlm, ltr); }

// ---------------------------------------------------------------------------
// Plan groups: scalar transforms of several plans (fields of different lmax,
// each on its own grid) where the Legendre stage of all plans is one
// persistent launch.  The per-plan prologue, FFT and epilogue launches fork
// from the stream of the first plan onto side streams of the group (one per
// plan) and join back before the persistent launch and at the end, all by
// events, so the small kernels of different plans run concurrently and the
// whole group stays one dependency graph rooted in the first plan's stream,
// which a CUDA graph captures as parallel branches.
// Work list of one direction (synthesis or analysis): per-plan parameters and
// (plan, order, tile, column tile) items, in pinned host memory and on the
// device.  The host copies are rewritten only after the stream has drained,
// so an upload still in flight never reads a half-written list, and each
// direction keeps its own buffers, so a captured graph holds both uploads
// (if any) with the right contents.
struct GroupWork {
	std::vector<int> key;            // field counts + ltr + order of the cached list
	LegParams* h_plist = nullptr; LegParams* d_plist = nullptr; int plist_cap = 0;
	int4* h_work = nullptr; int4* d_work = nullptr; int work_cap = 0; int nwork = 0;
	int* d_counter = nullptr;
	void release()
	{
		if (h_plist) cudaFreeHost(h_plist);
		if (d_plist) cudaFree(d_plist);
		if (h_work) cudaFreeHost(h_work);
		if (d_work) cudaFree(d_work);
		if (d_counter) cudaFree(d_counter);
		*this = GroupWork();
	}
};

struct shtns_b200_group {
	std::vector<shtns_cfg> plans;
	int ckseg;
	int order;                       // 0: work items by decreasing cost, 1: plan/order/tile order
	int nsm;
	int ctas_per_sm;                 // CTAs of the persistent launch per SM (1-3)
	int concurrent;                  // 1: per-plan launches on side streams (default), 0: all on the first plan's stream
	int leg_per_plan;                // 1: Legendre stage as each plan's own launch (concurrent); 0: one persistent launch
	GroupWork dir[2];                // [0] analysis, [1] synthesis
	std::vector<cudaStream_t> side;  // one per plan
	std::vector<cudaEvent_t> ev;     // fork + one join event per plan
};

namespace {

bool group_ok(shtns_group g)
{
	if (!g || g->plans.empty()) { shtb_set_error(1, "empty plan group"); return false; }
	return true;
}

// Runs launch(i, stream) for every plan i with fields: forked onto the
// group's side streams after the work already on st, joined back into st.
template <class F>
void group_fork(shtns_group g, cudaStream_t st, const int* nfields, F launch)
{
	const int np = (int) g->plans.size();
	if (!g->concurrent || (int) g->side.size() < np) {
		for (int i = 0; i < np; i++) if (nfields[i] > 0) launch(i, st);
		return;
	}
	cudaEventRecord(g->ev[0], st);
	for (int i = 0; i < np; i++) {
		if (nfields[i] <= 0) continue;
		cudaStreamWaitEvent(g->side[i], g->ev[0], 0);
		launch(i, g->side[i]);
		cudaEventRecord(g->ev[1 + i], g->side[i]);
	}
	for (int i = 0; i < np; i++)
		if (nfields[i] > 0) cudaStreamWaitEvent(st, g->ev[1 + i], 0);
}

// A list must change: refuse under stream capture (the host buffers would be
// read at replay time), else drain the stream so that no copy or kernel still
// uses the old list.
bool group_may_rewrite(cudaStream_t st)
{
	cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
	cudaStreamIsCapturing(st, &cs);
	if (cs != cudaStreamCaptureStatusNone) {
		shtb_set_error(1, "plan group: work list changed during stream capture "
		                  "(make one call with the same field counts before capturing)");
		return false;
	}
	return shtb_cuda_ok(cudaStreamSynchronize(st), "plan group stream");
}

// build (or reuse) the work list of the persistent Legendre launch
bool group_work(shtns_group g, const std::vector<LegParams>& lp, const int* nfields, bool synth)
{
	GroupWork& W = g->dir[synth ? 1 : 0];
	cudaStream_t st = g->plans[0]->comp_stream;
	const int np = (int) g->plans.size();
	std::vector<int> key;
	for (int i = 0; i < np; i++) { key.push_back(nfields[i]); key.push_back(lp[i].llim); }
	key.push_back(g->order);
	bool params_changed = W.plist_cap < np;
	for (int i = 0; i < np && !params_changed; i++)
		params_changed = memcmp(&W.h_plist[i], &lp[i], sizeof(LegParams)) != 0;
	const bool list_changed = key != W.key;
	if (!params_changed && !list_changed) return true;
	if (!group_may_rewrite(st)) return false;
	if (W.plist_cap < np) {
		if (W.h_plist) cudaFreeHost(W.h_plist);
		if (W.d_plist) cudaFree(W.d_plist);
		W.h_plist = nullptr; W.d_plist = nullptr; W.plist_cap = 0;
		if (cudaMallocHost(&W.h_plist, sizeof(LegParams) * np) != cudaSuccess ||
		    cudaMalloc(&W.d_plist, sizeof(LegParams) * np) != cudaSuccess) {
			cudaGetLastError(); shtb_set_error(3, "out of memory for plan group"); return false;
		}
		W.plist_cap = np;
	}
	if (!W.d_counter && cudaMalloc(&W.d_counter, sizeof(int)) != cudaSuccess) {
		cudaGetLastError(); shtb_set_error(3, "out of memory for plan group"); return false;
	}
	if (params_changed) {
		for (int i = 0; i < np; i++) W.h_plist[i] = lp[i];
		cudaMemcpyAsync(W.d_plist, W.h_plist, sizeof(LegParams) * np, cudaMemcpyHostToDevice, st);
	}
	if (!list_changed) return true;
	struct Item { int4 w; double cost; };
	std::vector<Item> items;
	for (int i = 0; i < np; i++) {
		if (nfields[i] <= 0) continue;
		const shtns_cfg s = g->plans[i];
		const LegParams& p = lp[i];
		const int nnb = (p.ncol + LG_BN - 1) / LG_BN;
		for (int im = 0; im <= p.mlim; im++) {
			const int m = im * s->mres;
			const int nk = (p.llim + p.vec_extra - m) / 2 + 1;
			const int tm = s->tm_h[im];
			if (synth) {
				const int ntb = (s->nlat_2 + LG_BM - 1) / LG_BM;
				for (int tb = 0; tb < ntb; tb++) {
					const bool live = tb * LG_BM + LG_BM > tm;
					const double cost = live ? (double) nk * LG_BM : 1.0;
					for (int nb = 0; nb < nnb; nb++) items.push_back({make_int4(i, im, tb, nb), cost});
				}
			} else {
				const int nkb = (nk + LG_BM - 1) / LG_BM;
				for (int kb = 0; kb < nkb; kb++) {
					const double cost = (double) (s->nlat_2 - (tm / LG_BK) * LG_BK) * std::min(LG_BM, nk - kb * LG_BM);
					for (int nb = 0; nb < nnb; nb++) items.push_back({make_int4(i, im, kb, nb), cost});
				}
			}
		}
	}
	if (g->order == 0)
		std::stable_sort(items.begin(), items.end(), [](const Item& a, const Item& b) { return a.cost > b.cost; });
	const int n = (int) items.size();
	if (W.work_cap < std::max(n, 1)) {
		if (W.h_work) cudaFreeHost(W.h_work);
		if (W.d_work) cudaFree(W.d_work);
		W.h_work = nullptr; W.d_work = nullptr; W.work_cap = 0;
		if (cudaMallocHost(&W.h_work, sizeof(int4) * std::max(n, 1)) != cudaSuccess ||
		    cudaMalloc(&W.d_work, sizeof(int4) * std::max(n, 1)) != cudaSuccess) {
			cudaGetLastError(); shtb_set_error(3, "out of memory for plan group"); W.key.clear(); return false;
		}
		W.work_cap = std::max(n, 1);
	}
	for (int i = 0; i < n; i++) W.h_work[i] = items[i].w;
	if (n > 0) cudaMemcpyAsync(W.d_work, W.h_work, sizeof(int4) * n, cudaMemcpyHostToDevice, st);
	W.nwork = n;
	W.key = key;
	return true;
}

} // namespace

extern "C" shtns_group shtns_b200_group_create(int nplans, shtns_cfg* plans)
{
	if (nplans < 1 || !plans) { shtb_set_error(1, "shtns_b200_group_create: no plans"); return nullptr; }
	int seg = plans[0] ? plans[0]->ckseg : 0;
	for (int i = 0; i < nplans; i++) {
		if (!plans[i] || !plans[i]->grid_set) { shtb_set_error(1, "shtns_b200_group_create: plan without grid"); return nullptr; }
		if (plans[i]->dev != plans[0]->dev) { shtb_set_error(1, "shtns_b200_group_create: plans on different devices"); return nullptr; }
		seg = std::max(seg, plans[i]->ckseg);
	}
	// one persistent kernel instance serves all plans: same checkpoint spacing
	for (int i = 0; i < nplans; i++)
		if (plans[i]->ckseg != seg && shtns_b200_set_option(plans[i], 2, seg) != 0) {
			shtb_set_error(1, "shtns_b200_group_create: cannot align checkpoint spacing");
			return nullptr;
		}
	shtns_group g = new shtns_b200_group();
	g->plans.assign(plans, plans + nplans);
	g->ckseg = seg;
	g->order = 0;
	g->ctas_per_sm = 3;
	g->concurrent = 1;
	cudaDeviceGetAttribute(&g->nsm, cudaDevAttrMultiProcessorCount, plans[0]->dev);
	g->side.assign(nplans, nullptr);
	g->ev.assign(nplans + 1, nullptr);
	bool ok = true;
	for (int i = 0; i < nplans && ok; i++) ok = cudaStreamCreateWithFlags(&g->side[i], cudaStreamNonBlocking) == cudaSuccess;
	for (int i = 0; i <= nplans && ok; i++) ok = cudaEventCreateWithFlags(&g->ev[i], cudaEventDisableTiming) == cudaSuccess;
	if (!ok) {
		// fall back to the single stream
		cudaGetLastError();
		for (cudaStream_t x : g->side) if (x) cudaStreamDestroy(x);
		for (cudaEvent_t e : g->ev) if (e) cudaEventDestroy(e);
		g->side.clear(); g->ev.clear();
		g->concurrent = 0;
	}
	return g;
}

extern "C" void shtns_b200_group_destroy(shtns_group g)
{
	if (!g) return;
	if (!g->plans.empty()) cudaStreamSynchronize(g->plans[0]->comp_stream);
	g->dir[0].release();
	g->dir[1].release();
	for (cudaStream_t x : g->side) if (x) cudaStreamDestroy(x);
	for (cudaEvent_t e : g->ev) if (e) cudaEventDestroy(e);
	delete g;
}

extern "C" int shtns_b200_group_set_option(shtns_group g, int option, int value)
{
	if (!g) return -1;
	if (option == 1 && (value == 0 || value == 1)) { g->order = value; return 0; }
	if (option == 2 && value >= 0 && value <= 3) { g->ctas_per_sm = value ? value : 3; return 0; }
	if (option == 5 && (value == 0 || value == 1)) { g->leg_per_plan = value; return 0; }
	if (option == 4 && (value == 0 || value == 1)) {
		if (value && g->side.empty()) return -1;     // no side streams: single-stream form only
		g->concurrent = value;
		return 0;
	}
	if (option == 3 && (value == 8 || value == 16 || value == 32)) {
		for (shtns_cfg s : g->plans)
			if (s->ckseg != value && shtns_b200_set_option(s, 2, value) != 0) return -1;
		g->ckseg = value;
		return 0;
	}
	return -1;
}

namespace {

// Group transforms of ncomp components (types: T_SCAL, T_VEC or T_QST): the
// spectral arrays spec[c][i] and the grids spat[c][i] of component c, plan i
// (a null array list reads zeros / is not written, as for the plan calls).
void group_synth_impl(shtns_group g, int ncomp, const int* types, cplx** const* spec, double** const* spat,
                      const int* nfields, int ltr)
{
	if (!group_ok(g)) return;
	const int np = (int) g->plans.size();
	cudaStream_t st = g->plans[0]->comp_stream;
	std::vector<Job> jobs(np);
	std::vector<LegParams> lp(np);
	for (int i = 0; i < np; i++) {
		shtns_cfg s = g->plans[i];
		shtns_set_batch(s, std::max(1, nfields[i]), s->nlm, s->nspat);
		if (!setup_job(s, jobs[i], ncomp, types, std::min<int>(ltr, s->lmax))) return;
		lp[i] = leg_params(s, jobs[i]);
	}
	auto prologue = [&](int i, cudaStream_t x) {
		PrepParams pp = prep_params(g->plans[i], jobs[i]);
		pp.Q = spec[0] ? reinterpret_cast<const double2*>(spec[0][i]) : nullptr;
		pp.S = spec[1] ? reinterpret_cast<const double2*>(spec[1][i]) : nullptr;
		pp.T = spec[2] ? reinterpret_cast<const double2*>(spec[2][i]) : nullptr;
		launch_prep_synth(pp, x);
	};
	auto fft = [&](int i, cudaStream_t x) {
		FftParams fp = fft_params(g->plans[i], jobs[i]);
		double* o[3];
		for (int c = 0; c < 3; c++) o[c] = (c < ncomp && spat[c]) ? spat[c][i] : nullptr;
		for (int c = 0; c < 3; c++) fp.spat[c] = o[c];
		fp.vec2 = aligned16(o[0], o[1] ? o[1] : o[0], o[2] ? o[2] : o[0], g->plans[i]->spat_dist);
		launch_fft_synth(fp, jobs[i].nfc, x);
	};
	if (g->leg_per_plan) {
		// each plan's own Legendre launch (its tile shape or SIMT kernels):
		// prologue, Legendre and FFT chained per plan on its side stream
		group_fork(g, st, nfields, [&](int i, cudaStream_t x) {
			prologue(i, x);
			launch_leg_synth(lp[i], x);
			fft(i, x);
		});
		check_launch("group synthesis launch");
		return;
	}
	if (!group_work(g, lp, nfields, true)) return;
	group_fork(g, st, nfields, prologue);
	const GroupWork& W = g->dir[1];
	launch_leg_multi(W.d_plist, W.d_work, W.nwork, W.d_counter, g->ckseg, true, g->nsm * g->ctas_per_sm, st);
	group_fork(g, st, nfields, fft);
	check_launch("group synthesis launch");
}

void group_analys_impl(shtns_group g, int ncomp, const int* types, double** const* spat, cplx** const* spec,
                       const int* nfields, int ltr)
{
	if (!group_ok(g)) return;
	const int np = (int) g->plans.size();
	cudaStream_t st = g->plans[0]->comp_stream;
	std::vector<Job> jobs(np);
	std::vector<LegParams> lp(np);
	for (int i = 0; i < np; i++) {
		shtns_cfg s = g->plans[i];
		shtns_set_batch(s, std::max(1, nfields[i]), s->nlm, s->nspat);
		if (!setup_job(s, jobs[i], ncomp, types, std::min<int>(ltr, s->lmax))) return;
		lp[i] = leg_params(s, jobs[i]);
	}
	auto fft = [&](int i, cudaStream_t x) {
		FftParams fp = fft_params(g->plans[i], jobs[i]);
		const double* in[3];
		for (int c = 0; c < 3; c++) in[c] = (c < ncomp && spat[c]) ? spat[c][i] : nullptr;
		for (int c = 0; c < 3; c++) fp.spat_in[c] = in[c];
		fp.vec2 = aligned16(in[0], in[1] ? in[1] : in[0], in[2] ? in[2] : in[0], g->plans[i]->spat_dist);
		launch_fft_analys(fp, jobs[i].nfc, x);
	};
	auto epilogue = [&](int i, cudaStream_t x) {
		PrepParams pp = prep_params(g->plans[i], jobs[i]);
		pp.Qo = spec[0] ? reinterpret_cast<double2*>(spec[0][i]) : nullptr;
		pp.So = spec[1] ? reinterpret_cast<double2*>(spec[1][i]) : nullptr;
		pp.To = spec[2] ? reinterpret_cast<double2*>(spec[2][i]) : nullptr;
		launch_post_analys_m(pp, g->plans[i]->mmax, x);
	};
	if (g->leg_per_plan) {
		group_fork(g, st, nfields, [&](int i, cudaStream_t x) {
			shtns_cfg s = g->plans[i];
			fft(i, x);
			int kmax_all = 0;
			for (int im = 0; im <= jobs[i].mlim; im++)
				kmax_all = std::max(kmax_all, (jobs[i].llim + jobs[i].vec_extra - im * s->mres) / 2 + 1);
			launch_leg_analys(lp[i], kmax_all, x);
			epilogue(i, x);
		});
		check_launch("group analysis launch");
		return;
	}
	if (!group_work(g, lp, nfields, false)) return;
	group_fork(g, st, nfields, fft);
	const GroupWork& W = g->dir[0];
	launch_leg_multi(W.d_plist, W.d_work, W.nwork, W.d_counter, g->ckseg, false, g->nsm * g->ctas_per_sm, st);
	group_fork(g, st, nfields, epilogue);
	check_launch("group analysis launch");
}

} // namespace

extern "C" void shtns_b200_group_synth(shtns_group g, cplx** Qlm, double** Vr, const int* nfields, int ltr)
{
	cplx** const spec[3] = {Qlm, nullptr, nullptr};
	double** const spat[3] = {Vr, nullptr, nullptr};
	group_synth_impl(g, 1, T_SCAL, spec, spat, nfields, ltr);
}

extern "C" void shtns_b200_group_analys(shtns_group g, double** Vr, cplx** Qlm, const int* nfields, int ltr)
{
	double** const spat[3] = {Vr, nullptr, nullptr};
	cplx** const spec[3] = {Qlm, nullptr, nullptr};
	group_analys_impl(g, 1, T_SCAL, spat, spec, nfields, ltr);
}

extern "C" void shtns_b200_group_SHsphtor_to_spat(shtns_group g, cplx** Slm, cplx** Tlm, double** Vt, double** Vp,
                                                  const int* nfields, int ltr)
{
	cplx** const spec[3] = {nullptr, Slm, Tlm};
	double** const spat[3] = {Vt, Vp, nullptr};
	group_synth_impl(g, 2, T_VEC, spec, spat, nfields, ltr);
}

extern "C" void shtns_b200_group_spat_to_SHsphtor(shtns_group g, double** Vt, double** Vp, cplx** Slm, cplx** Tlm,
                                                  const int* nfields, int ltr)
{
	double** const spat[3] = {Vt, Vp, nullptr};
	cplx** const spec[3] = {nullptr, Slm, Tlm};
	group_analys_impl(g, 2, T_VEC, spat, spec, nfields, ltr);
}

extern "C" void shtns_b200_group_SHqst_to_spat(shtns_group g, cplx** Qlm, cplx** Slm, cplx** Tlm, double** Vr, double** Vt,
                                               double** Vp, const int* nfields, int ltr)
{
	cplx** const spec[3] = {Qlm, Slm, Tlm};
	double** const spat[3] = {Vr, Vt, Vp};
	group_synth_impl(g, 3, T_QST, spec, spat, nfields, ltr);
}

extern "C" void shtns_b200_group_spat_to_SHqst(shtns_group g, double** Vr, double** Vt, double** Vp, cplx** Qlm, cplx** Slm,
                                               cplx** Tlm, const int* nfields, int ltr)
{
	double** const spat[3] = {Vr, Vt, Vp};
	cplx** const spec[3] = {Qlm, Slm, Tlm};
	group_analys_impl(g, 3, T_QST, spat, spec, nfields, ltr);
}

// ---------------------------------------------------------------------------
// Legendre transforms of one order m = |im|*mres, no FFT (shtns.h:329-342,
// sht_com.c:95-126; a negative im changes the sign of m in the vector terms,
// fly_SH_to_spat.gen.c:294-296).  Host arrays: spectral lmax+1-m complex coefficients of
// that order, spatial nlat complex values (the order's Fourier coefficient
// per grid row: v = sum_m (2 - delta_m0) Re(V_m e^{i m phi})).  The pipeline
// is the whole transform's prologue, Legendre and epilogue kernels launched
// for the single order (im0 = mlim = im), with the plan's Fourier buffer as
// the spatial side.
namespace {

long lm_first(shtns_cfg s, int im)   // LM(m, m), shtns.h:104-106
{
	return (long) im * (2 * s->lmax + 2 - (im + 1) * s->mres) / 2 + (long) im * s->mres;
}

template <class T> T* shifted(T* p, long n)   // p - n elements, for base[off + d] addressing
{
	return p ? reinterpret_cast<T*>(reinterpret_cast<uintptr_t>(p) - n * (long) sizeof(T)) : nullptr;
}

bool ml_job(shtns_cfg s, int im, int ncomp, const int* types, int ltr, Job& j)
{
	if (!s || !s->grid_set) { shtb_set_error(1, "transform on a plan without grid"); return false; }
	if (im > s->mmax || -im > s->mmax) { shtb_set_error(1, "fixed-order transform: order index out of range"); return false; }
	const int saved = s->batch;
	s->batch = 1;
	const bool ok = setup_job(s, j, ncomp, types, ltr);
	s->batch = saved;
	return ok;
}

void ml_synth(shtns_cfg s, int im, int ncomp, const int* types, const cplx* Q, const cplx* S, const cplx* T,
              cplx* o0, cplx* o1, cplx* o2, int ltr)
{
	Job j;
	if (!ml_job(s, im, ncomp, types, ltr, j)) return;
	const int msign = im < 0 ? -1 : 1;           // scalar terms use |m|, vector terms the signed m
	im = im < 0 ? -im : im;
	const int m = im * s->mres, nl = s->lmax + 1 - m;
	cplx* outs[3] = {o0, o1, o2};
	if (m > j.llim) {
		for (int c = 0; c < ncomp; c++) memset(outs[c], 0, sizeof(cplx) * s->nlat);
		return;
	}
	cudaStream_t cs = s->comp_stream;
	size_t cap = s->stage_cap;
	if (!ensure(&s->d_stage, &cap, sizeof(double2) * 3 * (size_t) nl, "staging buffers")) { s->stage_cap = 0; return; }
	s->stage_cap = cap;
	double2* st = static_cast<double2*>(s->d_stage);
	const cplx* ins[3] = {Q, S, T};
	for (int c = 0; c < 3; c++)
		if (ins[c]) cudaMemcpyAsync(st + c * nl, ins[c], sizeof(double2) * nl, cudaMemcpyHostToDevice, cs);
	const long off = lm_first(s, im);
	PrepParams pp = prep_params(s, j);
	pp.im0 = im; pp.mlim = im; pp.spec_dist = nl; pp.msign = msign;
	pp.Q = Q ? shifted<const double2>(st, off) : nullptr;
	pp.S = S ? shifted<const double2>(st + nl, off) : nullptr;
	pp.T = T ? shifted<const double2>(st + 2 * nl, off) : nullptr;
	launch_prep_synth(pp, cs);
	LegParams lp = leg_params(s, j);
	lp.im0 = im; lp.mlim = im;
	launch_leg_synth(lp, cs);
	check_launch("fixed-order synthesis launch");
	const long fstride = (long)(s->mmax + 1) * s->nlat;
	for (int c = 0; c < ncomp; c++)
		cudaMemcpyAsync(outs[c], s->d_F + c * fstride + (long) im * s->nlat, sizeof(double2) * s->nlat,
		                cudaMemcpyDeviceToHost, cs);
	shtb_cuda_ok(cudaStreamSynchronize(cs), "fixed-order synthesis");
}

void ml_analys(shtns_cfg s, int im, int ncomp, const int* types, const cplx* i0, const cplx* i1, const cplx* i2,
               cplx* Qo, cplx* So, cplx* To, int ltr)
{
	Job j;
	if (!ml_job(s, im, ncomp, types, ltr, j)) return;
	const int msign = im < 0 ? -1 : 1;
	im = im < 0 ? -im : im;
	const int m = im * s->mres, nl = s->lmax + 1 - m;
	cplx* outs[3] = {Qo, So, To};
	if (m > j.llim) {
		for (int c = 0; c < 3; c++) if (outs[c]) memset(outs[c], 0, sizeof(cplx) * nl);
		return;
	}
	cudaStream_t cs = s->comp_stream;
	const long fstride = (long)(s->mmax + 1) * s->nlat;
	const cplx* ins[3] = {i0, i1, i2};
	for (int c = 0; c < ncomp; c++)
		cudaMemcpyAsync(s->d_F + c * fstride + (long) im * s->nlat, ins[c], sizeof(double2) * s->nlat,
		                cudaMemcpyHostToDevice, cs);
	LegParams lp = leg_params(s, j);
	lp.im0 = im; lp.mlim = im;
	launch_leg_analys(lp, (j.llim + j.vec_extra - m) / 2 + 1, cs);
	size_t cap = s->stage_cap;
	if (!ensure(&s->d_stage, &cap, sizeof(double2) * 3 * (size_t) nl, "staging buffers")) { s->stage_cap = 0; return; }
	s->stage_cap = cap;
	double2* st = static_cast<double2*>(s->d_stage);
	const long off = lm_first(s, im);
	PrepParams pp = prep_params(s, j);
	pp.im0 = im; pp.mlim = im; pp.spec_dist = nl; pp.msign = msign;
	pp.Qo = Qo ? shifted<double2>(st, off) : nullptr;
	pp.So = So ? shifted<double2>(st + nl, off) : nullptr;
	pp.To = To ? shifted<double2>(st + 2 * nl, off) : nullptr;
	launch_post_analys_m(pp, im, cs);
	check_launch("fixed-order analysis launch");
	for (int c = 0; c < 3; c++)
		if (outs[c]) cudaMemcpyAsync(outs[c], st + c * nl, sizeof(double2) * nl, cudaMemcpyDeviceToHost, cs);
	shtb_cuda_ok(cudaStreamSynchronize(cs), "fixed-order analysis");
}

} // namespace

extern "C" void SH_to_spat_ml(shtns_cfg s, int im, cplx* Ql, cplx* Vr, int ltr)
{ ml_synth(s, im, 1, T_SCAL, Ql, nullptr, nullptr, Vr, nullptr, nullptr, ltr); }

extern "C" void spat_to_SH_ml(shtns_cfg s, int im, cplx* Vr, cplx* Ql, int ltr)
{ ml_analys(s, im, 1, T_SCAL, Vr, nullptr, nullptr, Ql, nullptr, nullptr, ltr); }

extern "C" void SHsphtor_to_spat_ml(shtns_cfg s, int im, cplx* Sl, cplx* Tl, cplx* Vt, cplx* Vp, int ltr)
{ ml_synth(s, im, 2, T_VEC, nullptr, Sl, Tl, Vt, Vp, nullptr, ltr); }

extern "C" void spat_to_SHsphtor_ml(shtns_cfg s, int im, cplx* Vt, cplx* Vp, cplx* Sl, cplx* Tl, int ltr)
{ ml_analys(s, im, 2, T_VEC, Vt, Vp, nullptr, nullptr, Sl, Tl, ltr); }

extern "C" void SHsph_to_spat_ml(shtns_cfg s, int im, cplx* Sl, cplx* Vt, cplx* Vp, int ltr)
{ ml_synth(s, im, 2, T_VEC, nullptr, Sl, nullptr, Vt, Vp, nullptr, ltr); }

extern "C" void SHtor_to_spat_ml(shtns_cfg s, int im, cplx* Tl, cplx* Vt, cplx* Vp, int ltr)
{ ml_synth(s, im, 2, T_VEC, nullptr, nullptr, Tl, Vt, Vp, nullptr, ltr); }

extern "C" void SHqst_to_spat_ml(shtns_cfg s, int im, cplx* Ql, cplx* Sl, cplx* Tl, cplx* Vr, cplx* Vt, cplx* Vp, int ltr)
{ ml_synth(s, im, 3, T_QST, Ql, Sl, Tl, Vr, Vt, Vp, ltr); }

extern "C" void spat_to_SHqst_ml(shtns_cfg s, int im, cplx* Vr, cplx* Vt, cplx* Vp, cplx* Ql, cplx* Sl, cplx* Tl, int ltr)
{ ml_analys(s, im, 3, T_QST, Vr, Vt, Vp, Ql, Sl, Tl, ltr); }

// ---------------------------------------------------------------------------
// Complex-valued fields (shtns.h:268-309, sht_func.c:939-1210): z(theta, phi)
// = sum_{l, -l<=m<=l} alm[LM_cplx(l, m)] Y_l^m, mres = 1.  Built from the
// real-field pipeline with two fields per component: field A carries the
// orders +m (A_lm = alm[l, m]; at m = 0 the real part), field B the orders -m
// (B_lm = (-1)^m alm[l, -m], with -m in the vector terms; at m = 0 the
// imaginary part).  The Legendre stage gives Q_{+m} (rows of A) and Q_{-m}
// (rows of B); in Fourier space these become the order-m coefficients of
// x = Re z and y = Im z,
//   X_m = (Q_m + conj Q_{-m}) / 2,  Y_m = (-i Q_m + i conj Q_{-m}) / 2  (m > 0),
// which the real FFT turns into the grids x and y, interleaved into z.  The
// analysis runs the same steps backwards (Q_m = X_m + i Y_m,
// Q_{-m} = conj X_m + i conj Y_m).
namespace {

__device__ __forceinline__ long lm_real_idx(int lmax, int im, int l)        // LM(l, m), mres = 1
{
	return (long) im * (2 * lmax + 1 - im) / 2 + l;
}

__device__ __forceinline__ long lm_cplx_idx(int lmax, int mmax, int l, int m)   // LM_cplx(l, m), shtns.h:114
{
	return (l <= mmax) ? (long) l * (l + 1) + m : (long) mmax * (2 * l - mmax) + l + m;
}

// alm (ncomp arrays of nlm_cplx) -> AB[comp][field][nlm]; grid (l blocks, im, comp)
__global__ void cplx_gather_kernel(const double2* __restrict__ a0, const double2* __restrict__ a1,
                                   const double2* __restrict__ a2, double2* __restrict__ ab, int lmax, int mmax, long nlm)
{
	const int im = blockIdx.y, c = blockIdx.z;
	const int l = im + blockIdx.x * blockDim.x + threadIdx.x;
	if (l > lmax) return;
	const double2* a = (c == 0) ? a0 : (c == 1 ? a1 : a2);
	const double2 p = a[lm_cplx_idx(lmax, mmax, l, im)];
	double2 A, B;
	if (im == 0) { A = make_double2(p.x, 0.0); B = make_double2(p.y, 0.0); }
	else {
		const double2 n = a[lm_cplx_idx(lmax, mmax, l, -im)];
		A = p;
		B = (im & 1) ? make_double2(-n.x, -n.y) : n;
	}
	const long r = lm_real_idx(lmax, im, l);
	ab[(2L * c) * nlm + r] = A;
	ab[(2L * c + 1) * nlm + r] = B;
}

// AB -> alm (inverse of the gather)
__global__ void cplx_scatter_kernel(const double2* __restrict__ ab, double2* __restrict__ a0, double2* __restrict__ a1,
                                    double2* __restrict__ a2, int lmax, int mmax, long nlm)
{
	const int im = blockIdx.y, c = blockIdx.z;
	const int l = im + blockIdx.x * blockDim.x + threadIdx.x;
	if (l > lmax) return;
	double2* a = (c == 0) ? a0 : (c == 1 ? a1 : a2);
	const long r = lm_real_idx(lmax, im, l);
	const double2 A = ab[(2L * c) * nlm + r], B = ab[(2L * c + 1) * nlm + r];
	if (im == 0) { a[lm_cplx_idx(lmax, mmax, l, 0)] = make_double2(A.x, B.x); return; }
	a[lm_cplx_idx(lmax, mmax, l, im)] = A;
	a[lm_cplx_idx(lmax, mmax, l, -im)] = (im & 1) ? make_double2(-B.x, -B.y) : B;
}

// Fourier rows: (Q_m, Q_{-m}) <-> (X_m, Y_m), in place in the (A, B) slots
__global__ void cplx_fourier_kernel(double2* __restrict__ F, long fstride, int nlat, int mlim, int ncomp, int to_xy)
{
	const long n = (long)(mlim + 1) * nlat;
	const long e = (long) blockIdx.x * blockDim.x + threadIdx.x;
	const int c = blockIdx.y;
	if (e >= n || c >= ncomp) return;
	const int m = (int)(e / nlat);
	double2* pa = F + (2L * c) * fstride + e;
	double2* pb = F + (2L * c + 1) * fstride + e;
	const double2 a = *pa, b = *pb;
	if (m == 0) {
		*pa = make_double2(a.x, 0.0);
		*pb = make_double2(b.x, 0.0);
	} else if (to_xy) {      // a = Q_m, b = Q_{-m}
		*pa = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
		*pb = make_double2(0.5 * (a.y + b.y), 0.5 * (b.x - a.x));
	} else {                 // a = X_m, b = Y_m
		*pa = make_double2(a.x - b.y, a.y + b.x);
		*pb = make_double2(a.x + b.y, b.x - a.y);
	}
}

// z[i] = (x[i], y[i]) and back; grid (blocks over nspat, comp)
__global__ void cplx_interleave_kernel(double2* __restrict__ z, long zdist, double* __restrict__ xy, long nspat, int to_z)
{
	const long i = (long) blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nspat) return;
	const int c = blockIdx.y;
	double* x = xy + (2L * c) * nspat;
	double* y = x + nspat;
	double2* zc = z + c * zdist;
	if (to_z) zc[i] = make_double2(x[i], y[i]);
	else { const double2 v = zc[i]; x[i] = v.x; y[i] = v.y; }
}

struct CplxStage {
	double2* alm;       // ncomp x nlm_cplx
	double2* ab;        // ncomp x 2 x nlm
	double* xy;         // ncomp x 2 x nspat
	double2* z;         // ncomp x nspat
};

bool cplx_begin(shtns_cfg s, int ncomp, const int* types, Job& j, CplxStage& cs)
{
	if (!s || !s->grid_set) { shtb_set_error(1, "transform on a plan without grid"); return false; }
	if (s->mres != 1) { shtb_set_error(1, "complex-valued transforms require mres = 1"); return false; }
	const int saved = s->batch;
	s->batch = 2;
	const bool ok = setup_job(s, j, ncomp, types, s->lmax);
	s->batch = saved;
	if (!ok) return false;
	const size_t nlmc = (size_t) s->nlm_cplx, nlm = s->nlm, nspat = s->nspat;
	auto al = [](size_t b) { return (b + 255) & ~(size_t) 255; };
	const size_t b_alm = al(sizeof(double2) * ncomp * nlmc), b_ab = al(sizeof(double2) * ncomp * 2 * nlm);
	const size_t b_xy = al(sizeof(double) * ncomp * 2 * nspat), b_z = al(sizeof(double2) * ncomp * nspat);
	size_t cap = s->stage_cap;
	if (!ensure(&s->d_stage, &cap, b_alm + b_ab + b_xy + b_z, "staging buffers")) { s->stage_cap = 0; return false; }
	s->stage_cap = cap;
	char* b = static_cast<char*>(s->d_stage);
	cs.alm = reinterpret_cast<double2*>(b);
	cs.ab = reinterpret_cast<double2*>(b + b_alm);
	cs.xy = reinterpret_cast<double*>(b + b_alm + b_ab);
	cs.z = reinterpret_cast<double2*>(b + b_alm + b_ab + b_xy);
	return true;
}

void cplx_synth(shtns_cfg s, int ncomp, const int* types, const cplx* const* alm, cplx* const* z)
{
	Job j;
	CplxStage cs;
	if (!cplx_begin(s, ncomp, types, j, cs)) return;
	cudaStream_t st = s->comp_stream;
	const long nlmc = s->nlm_cplx, nlm = s->nlm, nspat = s->nspat;
	for (int c = 0; c < ncomp; c++)
		cudaMemcpyAsync(cs.alm + c * nlmc, alm[c], sizeof(double2) * nlmc, cudaMemcpyHostToDevice, st);
	dim3 gg((s->lmax + 1 + 127) / 128, s->mmax + 1, ncomp);
	cplx_gather_kernel<<<gg, 128, 0, st>>>(cs.alm, cs.alm + nlmc, cs.alm + 2 * nlmc, cs.ab, s->lmax, s->mmax, nlm);
	shtb_count_launch();
	PrepParams pp = prep_params(s, j);
	pp.spec_dist = nlm; pp.neg_from = 1;
	const double2* comps[3] = {cs.ab, cs.ab + 2 * nlm, cs.ab + 4 * nlm};
	if (ncomp == 1) pp.Q = comps[0];
	else if (ncomp == 2) { pp.S = comps[0]; pp.T = comps[1]; }
	else { pp.Q = comps[0]; pp.S = comps[1]; pp.T = comps[2]; }
	launch_prep_synth(pp, st);
	LegParams lp = leg_params(s, j);
	launch_leg_synth(lp, st);
	const long fstride = (long)(s->mmax + 1) * s->nlat;
	dim3 gf((unsigned)(((long)(j.mlim + 1) * s->nlat + 255) / 256), ncomp);
	cplx_fourier_kernel<<<gf, 256, 0, st>>>(s->d_F, fstride, s->nlat, j.mlim, ncomp, 1);
	shtb_count_launch();
	FftParams fp = fft_params(s, j);
	fp.spat_dist = nspat;
	for (int c = 0; c < ncomp; c++) fp.spat[c] = cs.xy + 2L * c * nspat;
	fp.vec2 = aligned16(fp.spat[0], fp.spat[ncomp > 1 ? 1 : 0], fp.spat[ncomp > 2 ? 2 : 0], nspat);
	launch_fft_synth(fp, j.nfc, st);
	dim3 gi((unsigned)((nspat + 255) / 256), ncomp);
	cplx_interleave_kernel<<<gi, 256, 0, st>>>(cs.z, nspat, cs.xy, nspat, 1);
	shtb_count_launch();
	check_launch("complex synthesis launch");
	for (int c = 0; c < ncomp; c++)
		cudaMemcpyAsync(z[c], cs.z + c * nspat, sizeof(double2) * nspat, cudaMemcpyDeviceToHost, st);
	shtb_cuda_ok(cudaStreamSynchronize(st), "complex synthesis");
}

void cplx_analys(shtns_cfg s, int ncomp, const int* types, const cplx* const* z, cplx* const* alm)
{
	Job j;
	CplxStage cs;
	if (!cplx_begin(s, ncomp, types, j, cs)) return;
	cudaStream_t st = s->comp_stream;
	const long nlmc = s->nlm_cplx, nlm = s->nlm, nspat = s->nspat;
	for (int c = 0; c < ncomp; c++)
		cudaMemcpyAsync(cs.z + c * nspat, z[c], sizeof(double2) * nspat, cudaMemcpyHostToDevice, st);
	dim3 gi((unsigned)((nspat + 255) / 256), ncomp);
	cplx_interleave_kernel<<<gi, 256, 0, st>>>(cs.z, nspat, cs.xy, nspat, 0);
	shtb_count_launch();
	FftParams fp = fft_params(s, j);
	fp.spat_dist = nspat;
	for (int c = 0; c < ncomp; c++) fp.spat_in[c] = cs.xy + 2L * c * nspat;
	fp.vec2 = aligned16(fp.spat_in[0], fp.spat_in[ncomp > 1 ? 1 : 0], fp.spat_in[ncomp > 2 ? 2 : 0], nspat);
	launch_fft_analys(fp, j.nfc, st);
	const long fstride = (long)(s->mmax + 1) * s->nlat;
	dim3 gf((unsigned)(((long)(j.mlim + 1) * s->nlat + 255) / 256), ncomp);
	cplx_fourier_kernel<<<gf, 256, 0, st>>>(s->d_F, fstride, s->nlat, j.mlim, ncomp, 0);
	shtb_count_launch();
	LegParams lp = leg_params(s, j);
	int kmax_all = 0;
	for (int im = 0; im <= j.mlim; im++) kmax_all = std::max(kmax_all, (j.llim + j.vec_extra - im) / 2 + 1);
	launch_leg_analys(lp, kmax_all, st);
	PrepParams pp = prep_params(s, j);
	pp.spec_dist = nlm; pp.neg_from = 1;
	double2* comps[3] = {cs.ab, cs.ab + 2 * nlm, cs.ab + 4 * nlm};
	if (ncomp == 1) pp.Qo = comps[0];
	else if (ncomp == 2) { pp.So = comps[0]; pp.To = comps[1]; }
	else { pp.Qo = comps[0]; pp.So = comps[1]; pp.To = comps[2]; }
	launch_post_analys_m(pp, s->mmax, st);
	dim3 gg((s->lmax + 1 + 127) / 128, s->mmax + 1, ncomp);
	cplx_scatter_kernel<<<gg, 128, 0, st>>>(cs.ab, cs.alm, cs.alm + nlmc, cs.alm + 2 * nlmc, s->lmax, s->mmax, nlm);
	shtb_count_launch();
	check_launch("complex analysis launch");
	for (int c = 0; c < ncomp; c++)
		cudaMemcpyAsync(alm[c], cs.alm + c * nlmc, sizeof(double2) * nlmc, cudaMemcpyDeviceToHost, st);
	shtb_cuda_ok(cudaStreamSynchronize(st), "complex analysis");
}

} // namespace

extern "C" void SH_to_spat_cplx(shtns_cfg s, cplx* alm, cplx* z)
{ const cplx* a[1] = {alm}; cplx* o[1] = {z}; cplx_synth(s, 1, T_SCAL, a, o); }

extern "C" void spat_cplx_to_SH(shtns_cfg s, cplx* z, cplx* alm)
{ const cplx* i[1] = {z}; cplx* o[1] = {alm}; cplx_analys(s, 1, T_SCAL, i, o); }

extern "C" void SHsphtor_to_spat_cplx(shtns_cfg s, cplx* Slm, cplx* Tlm, cplx* Vt, cplx* Vp)
{ const cplx* a[2] = {Slm, Tlm}; cplx* o[2] = {Vt, Vp}; cplx_synth(s, 2, T_VEC, a, o); }

extern "C" void spat_cplx_to_SHsphtor(shtns_cfg s, cplx* Vt, cplx* Vp, cplx* Slm, cplx* Tlm)
{ const cplx* i[2] = {Vt, Vp}; cplx* o[2] = {Slm, Tlm}; cplx_analys(s, 2, T_VEC, i, o); }

extern "C" void SHqst_to_spat_cplx(shtns_cfg s, cplx* Qlm, cplx* Slm, cplx* Tlm, cplx* Vr, cplx* Vt, cplx* Vp)
{ const cplx* a[3] = {Qlm, Slm, Tlm}; cplx* o[3] = {Vr, Vt, Vp}; cplx_synth(s, 3, T_QST, a, o); }

extern "C" void spat_cplx_to_SHqst(shtns_cfg s, cplx* Vr, cplx* Vt, cplx* Vp, cplx* Qlm, cplx* Slm, cplx* Tlm)
{ const cplx* i[3] = {Vr, Vt, Vp}; cplx* o[3] = {Qlm, Slm, Tlm}; cplx_analys(s, 3, T_QST, i, o); }

// ---------------------------------------------------------------------------
// Order-split stages: one transform divided over processes by order.  The
// Legendre stages work on a range of orders m0..m1 over every grid row, the
// Fourier (phi FFT) stages on a block of rows over every order; between them
// the caller moves Fourier rows so that each process holds what its next stage
// needs (an all-to-all when the processes are GPUs).  Buffers and pointers are
// device memory; every call is enqueued on the plan's compute stream.
//   Legendre-side Fourier buffer:  F[fc][im - m0][row], rows 0..nlat-1
//   Fourier-side Fourier buffer:   F[fc][im][r], im 0..mmax, r 0..nrows-1
// with fc = c * howmany + f for component c of field f.  Spatial blocks hold
// nrows consecutive grid rows of each field in the plan's layout with nrows in
// place of nlat (fields nphi*nrows doubles apart).  Spectral arrays keep the
// plan's full layout (field stride spec_dist); only orders m0..m1 are read or
// written.  Orders above the truncation ltr are not written on the Fourier
// side and not read by the FFT; the Legendre analysis writes them as zero.
namespace {

bool kind_types(int kind, int* ncomp, const int** types)
{
	switch (kind) {
		case 0: *ncomp = 1; *types = T_SCAL; return true;
		case 1: *ncomp = 2; *types = T_VEC; return true;
		case 2: *ncomp = 3; *types = T_QST; return true;
		default: shtb_set_error(1, "order-split stage: kind must be 0 (scalar), 1 (sphtor) or 2 (qst)"); return false;
	}
}

bool range_ok(shtns_cfg s, int m0, int m1, const void* F)
{
	if (m0 < 0 || m1 < m0 || m1 > s->mmax) { shtb_set_error(1, "order-split stage: invalid order range"); return false; }
	if (!F) { shtb_set_error(1, "order-split stage: null Fourier buffer"); return false; }
	return true;
}

bool rows_ok(shtns_cfg s, int nrows, const void* F)
{
	if (nrows <= 0 || nrows > (int) s->nlat || (nrows & 1)) {
		shtb_set_error(1, "order-split stage: row count must be even and in 2..nlat");
		return false;
	}
	if (!F) { shtb_set_error(1, "order-split stage: null Fourier buffer"); return false; }
	return true;
}

} // namespace

extern "C" void shtns_b200_legendre_synth(shtns_cfg s, int kind, cplx* Q, cplx* S, cplx* T, cplx* F,
                                          int m0, int m1, int ltr)
{
	int nc; const int* ty;
	Job j;
	if (!kind_types(kind, &nc, &ty) || !setup_job(s, j, nc, ty, ltr, 1) || !range_ok(s, m0, m1, F)) return;
	if (m0 > j.mlim) return;
	const int mhi = std::min(m1, j.mlim);
	PrepParams pp = prep_params(s, j);
	pp.im0 = m0; pp.mlim = mhi;
	pp.Q = reinterpret_cast<const double2*>(Q);
	pp.S = reinterpret_cast<const double2*>(S);
	pp.T = reinterpret_cast<const double2*>(T);
	shtb_stage_begin(s, 0);
	launch_prep_synth(pp, s->comp_stream);
	shtb_stage_end(s);
	LegParams lp = leg_params(s, j);
	lp.im0 = m0; lp.mlim = mhi;
	lp.F = shifted(reinterpret_cast<double2*>(F), (long) m0 * s->nlat);
	lp.fstride = (long)(m1 - m0 + 1) * s->nlat;
	shtb_stage_begin(s, 1);
	launch_leg_synth(lp, s->comp_stream);
	shtb_stage_end(s);
	check_launch("order-split Legendre synthesis launch");
}

extern "C" void shtns_b200_fourier_synth(shtns_cfg s, int kind, cplx* F, double* V0, double* V1, double* V2,
                                         int nrows, int ltr)
{
	int nc; const int* ty;
	Job j;
	if (!kind_types(kind, &nc, &ty) || !setup_job(s, j, nc, ty, ltr, 0) || !rows_ok(s, nrows, F)) return;
	FftParams fp = fft_params(s, j, nrows);
	fp.nlat = nrows;
	fp.F = reinterpret_cast<double2*>(F);
	fp.fstride = (long)(s->mmax + 1) * nrows;
	fp.spat_dist = (long) s->nphi * nrows;
	fp.spat[0] = V0; fp.spat[1] = V1; fp.spat[2] = V2;
	fp.vec2 = aligned16(V0, V1, V2, fp.spat_dist);
	shtb_stage_begin(s, 2);
	launch_fft_synth(fp, j.nfc, s->comp_stream);
	shtb_stage_end(s);
	check_launch("order-split FFT synthesis launch");
}

extern "C" void shtns_b200_fourier_analys(shtns_cfg s, int kind, double* V0, double* V1, double* V2, cplx* F,
                                          int nrows, int ltr)
{
	int nc; const int* ty;
	Job j;
	if (!kind_types(kind, &nc, &ty) || !setup_job(s, j, nc, ty, ltr, 0) || !rows_ok(s, nrows, F)) return;
	FftParams fp = fft_params(s, j, nrows);
	fp.nlat = nrows;
	fp.F = reinterpret_cast<double2*>(F);
	fp.fstride = (long)(s->mmax + 1) * nrows;
	fp.spat_dist = (long) s->nphi * nrows;
	fp.spat_in[0] = V0; fp.spat_in[1] = V1; fp.spat_in[2] = V2;
	fp.vec2 = aligned16(V0, V1, V2, fp.spat_dist);
	shtb_stage_begin(s, 3);
	launch_fft_analys(fp, j.nfc, s->comp_stream);
	shtb_stage_end(s);
	check_launch("order-split FFT analysis launch");
}

extern "C" void shtns_b200_legendre_analys(shtns_cfg s, int kind, cplx* F, cplx* Q, cplx* S, cplx* T,
                                           int m0, int m1, int ltr)
{
	int nc; const int* ty;
	Job j;
	if (!kind_types(kind, &nc, &ty) || !setup_job(s, j, nc, ty, ltr, 1) || !range_ok(s, m0, m1, F)) return;
	if (m0 <= j.mlim) {
		LegParams lp = leg_params(s, j);
		lp.im0 = m0; lp.mlim = std::min(m1, j.mlim);
		lp.F = shifted(reinterpret_cast<double2*>(F), (long) m0 * s->nlat);
		lp.fstride = (long)(m1 - m0 + 1) * s->nlat;
		shtb_stage_begin(s, 4);
		launch_leg_analys(lp, (j.llim + j.vec_extra - m0 * s->mres) / 2 + 1, s->comp_stream);
		shtb_stage_end(s);
	}
	PrepParams pp = prep_params(s, j);
	pp.im0 = m0;
	pp.Qo = reinterpret_cast<double2*>(Q);
	pp.So = reinterpret_cast<double2*>(S);
	pp.To = reinterpret_cast<double2*>(T);
	shtb_stage_begin(s, 5);
	launch_post_analys_m(pp, m1, s->comp_stream);
	shtb_stage_end(s);
	check_launch("order-split Legendre analysis launch");
}

// ---------------------------------------------------------------------------
// Order-split stages with the exchange fused into the Legendre kernels: the
// synthesis stores each Fourier row straight into the buffer of the block of
// grid rows that owns it (blocks lat0[b] .. lat0[b+1]-1, buffer F[b] laid out
// as the Fourier side of shtns_b200_fourier_synth), and the analysis loads
// the rows from there.  When the buffers are other GPUs' memory mapped into
// this process (shtns_b200_ipc_open), the stores and loads go over NVLink
// inside the Legendre kernels and no separate all-to-all remains.
namespace {

bool row_blocks(shtns_cfg s, int nblk, const int* lat0, cplx* const* F, RowBlocks& rb)
{
	if (nblk < 1 || nblk > SHTB_MAX_BLOCKS || !lat0 || !F) {
		shtb_set_error(1, "order-split rows: 1 to 16 blocks with row bounds and buffers required");
		return false;
	}
	memset(&rb, 0, sizeof(rb));
	rb.n = nblk;
	rb.mstride = s->mmax + 1;
	for (int b = 0; b <= nblk; b++) rb.lat0[b] = lat0[b];
	if (rb.lat0[0] != 0 || rb.lat0[nblk] != (int) s->nlat) {
		shtb_set_error(1, "order-split rows: blocks must cover rows 0..nlat-1");
		return false;
	}
	for (int b = 0; b < nblk; b++) {
		if (rb.lat0[b + 1] <= rb.lat0[b] || !F[b]) { shtb_set_error(1, "order-split rows: empty block or null buffer"); return false; }
		rb.base[b] = reinterpret_cast<double2*>(F[b]);
	}
	return true;
}

} // namespace

extern "C" void shtns_b200_legendre_synth_rows(shtns_cfg s, int kind, cplx* Q, cplx* S, cplx* T, int m0, int m1, int ltr,
                                               int nblk, const int* lat0, cplx** F)
{
	int nc; const int* ty;
	Job j;
	RowBlocks rb;
	if (!kind_types(kind, &nc, &ty) || !setup_job(s, j, nc, ty, ltr, 1)) return;
	if (m0 < 0 || m1 < m0 || m1 > s->mmax) { shtb_set_error(1, "order-split stage: invalid order range"); return; }
	if (!row_blocks(s, nblk, lat0, F, rb)) return;
	if (m0 > j.mlim) return;
	const int mhi = std::min(m1, j.mlim);
	PrepParams pp = prep_params(s, j);
	pp.im0 = m0; pp.mlim = mhi;
	pp.Q = reinterpret_cast<const double2*>(Q);
	pp.S = reinterpret_cast<const double2*>(S);
	pp.T = reinterpret_cast<const double2*>(T);
	shtb_stage_begin(s, 0);
	launch_prep_synth(pp, s->comp_stream);
	shtb_stage_end(s);
	LegParams lp = leg_params(s, j);
	lp.im0 = m0; lp.mlim = mhi;
	lp.rb = rb;
	shtb_stage_begin(s, 1);
	launch_leg_synth(lp, s->comp_stream);
	shtb_stage_end(s);
	check_launch("order-split Legendre synthesis launch");
}

extern "C" void shtns_b200_legendre_analys_rows(shtns_cfg s, int kind, int nblk, const int* lat0, cplx** F,
                                                cplx* Q, cplx* S, cplx* T, int m0, int m1, int ltr)
{
	int nc; const int* ty;
	Job j;
	RowBlocks rb;
	if (!kind_types(kind, &nc, &ty) || !setup_job(s, j, nc, ty, ltr, 1)) return;
	if (m0 < 0 || m1 < m0 || m1 > s->mmax) { shtb_set_error(1, "order-split stage: invalid order range"); return; }
	if (!row_blocks(s, nblk, lat0, F, rb)) return;
	if (m0 <= j.mlim) {
		LegParams lp = leg_params(s, j);
		lp.im0 = m0; lp.mlim = std::min(m1, j.mlim);
		lp.rb = rb;
		shtb_stage_begin(s, 4);
		launch_leg_analys(lp, (j.llim + j.vec_extra - m0 * s->mres) / 2 + 1, s->comp_stream);
		shtb_stage_end(s);
	}
	PrepParams pp = prep_params(s, j);
	pp.im0 = m0;
	pp.Qo = reinterpret_cast<double2*>(Q);
	pp.So = reinterpret_cast<double2*>(S);
	pp.To = reinterpret_cast<double2*>(T);
	shtb_stage_begin(s, 5);
	launch_post_analys_m(pp, m1, s->comp_stream);
	shtb_stage_end(s);
	check_launch("order-split Legendre analysis launch");
}

// Device allocations of their own (an IPC handle maps a whole allocation).
extern "C" void* shtns_b200_alloc(size_t bytes)
{
	void* p = nullptr;
	if (!shtb_cuda_ok(cudaMalloc(&p, bytes), "device buffer")) return nullptr;
	return p;
}

extern "C" void shtns_b200_free(void* p)
{
	if (p) cudaFree(p);
}

// CUDA IPC: the 64-byte handle of a device allocation made in this process,
// and the mapping of another process's handle (peer access enabled lazily).
extern "C" int shtns_b200_ipc_handle(void* dev_ptr, void* handle64)
{
	cudaIpcMemHandle_t h;
	if (!dev_ptr || !handle64) { shtb_set_error(1, "ipc handle: null argument"); return -1; }
	if (!shtb_cuda_ok(cudaIpcGetMemHandle(&h, dev_ptr), "cudaIpcGetMemHandle")) return -1;
	static_assert(sizeof(h) == 64, "CUDA IPC handles are 64 bytes");
	memcpy(handle64, &h, sizeof(h));
	return 0;
}

extern "C" void* shtns_b200_ipc_open(const void* handle64)
{
	cudaIpcMemHandle_t h;
	void* p = nullptr;
	if (!handle64) { shtb_set_error(1, "ipc open: null handle"); return nullptr; }
	memcpy(&h, handle64, sizeof(h));
	if (!shtb_cuda_ok(cudaIpcOpenMemHandle(&p, h, cudaIpcMemLazyEnablePeerAccess), "cudaIpcOpenMemHandle")) return nullptr;
	return p;
}

extern "C" void shtns_b200_ipc_close(void* ptr)
{
	if (ptr) shtb_cuda_ok(cudaIpcCloseMemHandle(ptr), "cudaIpcCloseMemHandle");
}
