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

// Test hook behind shtns_b200_set_option(s, 9, byte): fills the static array
// of the current device with one byte value (0xFF gives NaN doubles), so that
// a test can show that no call reads scratch it did not write.  cudaMemset on
// the array's device address allocates nothing.
int shtb_noalloc_fill(int byte)
{
	int dev = -1;
	if (!shtb_cuda_ok(cudaGetDevice(&dev), "static scratch fill")) return -1;
	void* base = scratch_address(dev);
	if (!base) return -1;
	if (!shtb_cuda_ok(cudaMemset(base, byte & 0xFF, SHTB_STATIC_SCRATCH_BYTES), "static scratch fill")) return -1;
	return shtb_cuda_ok(cudaDeviceSynchronize(), "static scratch fill") ? 0 : -1;
}

extern "C" void cu_SH_to_spat_noalloc(shtns_cfg s, cplx* Qlm, double* Vr, int ltr)
{
	if (!s || !s->grid_set) { shtb_set_error(1, "transform on a plan without grid"); return; }
	if (s->split_ns) {
		shtb_set_error(1, "cu_SH_to_spat_noalloc: split-precision synthesis (plan option 4) needs tables and "
		                  "buffers allocated on first use; switch it off (option 4 = 0) for this entry point");
		return;
	}
	int dev = -1;
	if (!shtb_cuda_ok(cudaGetDevice(&dev), "cu_SH_to_spat_noalloc")) return;
	if (dev != s->dev) { shtb_set_error(1, "cu_SH_to_spat_noalloc: current device differs from the plan's device"); return; }
	// the call's shape with every plan option applied; bufs = 0: no plan buffer is grown
	static const int scalar_type[1] = {0};
	Job j;
	if (!setup_job(s, j, 1, scalar_type, ltr, 0)) return;
	const size_t qq_bytes = ((sizeof(double) * (size_t) s->ktot * j.ncol) + 255) & ~(size_t) 255;
	const size_t F_bytes = sizeof(double2) * (size_t) j.nfc * (s->mmax + 1) * s->nlat;
	if (qq_bytes + F_bytes > SHTB_STATIC_SCRATCH_BYTES) {
		shtb_set_error(1, "cu_SH_to_spat_noalloc: this plan and batch need " + std::to_string(qq_bytes + F_bytes) +
		                  " bytes of scratch, more than the static " + std::to_string(SHTB_STATIC_SCRATCH_BYTES) + " bytes");
		return;
	}
	void* base = scratch_address(dev);
	if (!base) return;
	double* qq = static_cast<double*>(base);
	double2* F = reinterpret_cast<double2*>(static_cast<char*>(base) + qq_bytes);

	PrepParams pp = prep_params(s, j);
	pp.Q = reinterpret_cast<const double2*>(Qlm);
	pp.qq = qq;
	LegParams lp = leg_params(s, j);
	lp.qq = qq; lp.F = F;
	FftParams fp = fft_params(s, j);
	fp.F = F;
	fp.spat[0] = Vr;
	fp.vec2 = (((uintptr_t) Vr & 15) == 0) && (s->spat_dist % 2 == 0);

	launch_prep_synth(pp, s->comp_stream);
	launch_leg_synth(lp, s->comp_stream);
	launch_fft_synth(fp, j.nfc, s->comp_stream);
	shtb_cuda_ok(cudaGetLastError(), "cu_SH_to_spat_noalloc launch");
}
