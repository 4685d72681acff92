// Scalar synthesis that allocates no device memory.
//
// Some callers cannot call cudaMalloc at the point where they transform:
// code that runs inside a region where allocation is forbidden (a real-time
// loop, an allocator-free plug-in host, or a process whose device memory is
// handed out by another component) and code that must not trigger the
// implicit synchronisation an allocation can cause.  cu_SH_to_spat grows
// plan-owned work buffers with cudaMalloc on first use; this entry point
// instead runs the same three kernels with their scratch (the Ishioka
// coefficient buffer and the Fourier buffer) placed in one file-scope static
// device array of SHTB_STATIC_SCRATCH_BYTES.  The plan tables are still made
// by shtns_set_grid, once, before the restricted region.
//
// The static array exists once per device that loads this library and stays
// allocated until the process exits.  All calls share it: two calls that
// overlap on the GPU (different streams, or different plans in flight at the
// same time) race on it and must be serialised by the caller.  No part of it
// needs to start at zero: every value a kernel reads was written earlier in
// the same call.
#include "sht_internal.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>

#define SHTB_STATIC_SCRATCH_BYTES (32u << 20)   // 32 MiB

static __device__ __align__(256) unsigned char g_static_scratch[SHTB_STATIC_SCRATCH_BYTES];

namespace {

std::mutex g_scratch_mu;
void* g_scratch_addr[128] = {nullptr};

// Device address of the static array on the current device.  In host code
// the name g_static_scratch is only a host-side stand-in, so the address is
// resolved once per device with cudaGetSymbolAddress (on the first call on
// that device; this may also make the runtime load this file's device code).
void* scratch_address(int dev)
{
	if (dev < 0 || dev >= 128) { shtb_set_error(1, "device id out of range"); return nullptr; }
	std::lock_guard<std::mutex> lk(g_scratch_mu);
	if (!g_scratch_addr[dev]) {
		void* ptr = nullptr;
		const cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_scratch);
		if (e != cudaSuccess || ptr == nullptr) {
			shtb_set_error(2, std::string("cudaGetSymbolAddress of the static scratch failed: ") + cudaGetErrorString(e));
			return nullptr;
		}
		g_scratch_addr[dev] = ptr;
	}
	return g_scratch_addr[dev];
}

} // namespace

extern "C" void cu_SH_to_spat_noalloc(shtns_cfg s, cplx* Qlm, double* Vr, int ltr)
{
	if (!s || !s->grid_set) { shtb_set_error(1, "transform on a plan without grid"); return; }
	if (ltr < 0) { shtb_set_error(1, "negative truncation degree"); return; }
	int dev = -1;
	if (!shtb_cuda_ok(cudaGetDevice(&dev), "cu_SH_to_spat_noalloc")) return;
	if (dev != s->dev) { shtb_set_error(1, "cu_SH_to_spat_noalloc: current device differs from the plan's device"); return; }
	const int nf = s->batch;
	const int nfc = nf;
	const int ncol = 16 * ((nfc + 3) / 4);
	const int llim = std::min<int>(ltr, s->lmax);
	const int mlim = std::min<int>(s->mmax, llim / s->mres);
	const size_t qq_bytes = ((sizeof(double) * (size_t) s->ktot * ncol) + 255) & ~(size_t) 255;
	const size_t F_bytes = sizeof(double2) * (size_t) nfc * (s->mmax + 1) * s->nlat;
	if (qq_bytes + F_bytes > SHTB_STATIC_SCRATCH_BYTES) {
		shtb_set_error(1, "cu_SH_to_spat_noalloc: this plan and batch need " + std::to_string(qq_bytes + F_bytes) +
		                  " bytes of scratch, more than the static " + std::to_string(SHTB_STATIC_SCRATCH_BYTES) + " bytes");
		return;
	}
	void* base = scratch_address(dev);
	if (!base) return;
	double* qq = static_cast<double*>(base);
	double2* F = reinterpret_cast<double2*>(static_cast<char*>(base) + qq_bytes);

	PrepParams pp;
	memset(&pp, 0, sizeof(pp));
	pp.lmax = s->lmax; pp.llim = llim; pp.mlim = mlim; pp.mres = s->mres;
	pp.nf = nf; pp.ncomp = 1; pp.ncol = ncol;
	pp.spec_dist = s->spec_dist;
	pp.xs = s->d_xs; pp.xa = s->d_xa;
	pp.stdt_lo = s->d_stdt_lo; pp.stdt_hi = s->d_stdt_hi; pp.van_lo = s->d_van_lo; pp.van_hi = s->d_van_hi;
	pp.l2 = s->d_l2; pp.mt = s->mt; pp.qq = qq;
	pp.Q = reinterpret_cast<const double2*>(Qlm);

	LegParams lp;
	memset(&lp, 0, sizeof(lp));
	lp.nlat = s->nlat; lp.nlat_2 = s->nlat_2; lp.llim = llim; lp.mlim = mlim; lp.mres = s->mres;
	lp.vec_extra = 0; lp.ncol = ncol; lp.nfc = nfc; lp.ckseg = s->ckseg;
	lp.south_first = s->south_first; lp.robert = s->robert;
	lp.mpos_inv = 1.0 / s->mpos_renorm;
	lp.x = s->d_x; lp.x2 = s->d_x2; lp.sinv = s->d_sinv; lp.w = s->d_w; lp.c = s->d_c;
	lp.ck = s->d_ck; lp.mt = s->mt; lp.nf = nf;
	lp.qq = qq; lp.F = F;
	lp.fstride = (long)(s->mmax + 1) * s->nlat;

	FftParams fp;
	memset(&fp, 0, sizeof(fp));
	fp.N = s->nphi; fp.nlat = s->nlat; fp.mlim = mlim;
	fp.nradix = (int) s->fft_radix.size();
	for (int i = 0; i < fp.nradix; i++) fp.rcode |= (unsigned long long) s->fft_radix[i] << (4 * i);
	int S = 4;
	while (S > 1 && fft_smem_bytes(s->nphi, S) > 112 * 1024) S /= 2;
	while (S > 1 && 2 * S > (int) s->nlat) S /= 2;
	fp.S = S;
	fp.tw = s->d_tw; fp.F = F;
	fp.fstride = lp.fstride;
	fp.nf = nf; fp.spat_dist = s->spat_dist;
	fp.phi_contiguous = s->phi_contiguous;
	fp.spat[0] = Vr;
	fp.vec2 = (((uintptr_t) Vr & 15) == 0) && (s->spat_dist % 2 == 0);

	launch_prep_synth(pp, s->comp_stream);
	launch_leg_synth(lp, s->comp_stream);
	launch_fft_synth(fp, nfc, s->comp_stream);
	shtb_cuda_ok(cudaGetLastError(), "cu_SH_to_spat_noalloc launch");
}
