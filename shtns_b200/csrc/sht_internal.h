// Private definitions of shtns_b200: the plan structure, the per-order (m)
// table layout in GPU memory and the kernel launch interfaces.
#pragma once

#define SHTNS_B200_PRIVATE
#include "../../include/shtns.h"
#include "../../include/shtns_cuda.h"
#include "../../include/shtns_b200.h"

#include <cuda_runtime.h>
#include <vector>
#include <string>
#include <cstdint>

// Tile sizes of the Legendre contraction kernels (see sht_legendre.cu).
#define LG_BM 64      // synthesis: theta rows per CTA;  analysis: k rows per CTA
#define LG_BN 64      // real columns per CTA (16 field-components x {E,O} x {re,im})
#define LG_BK 32      // synthesis: k per chunk;  analysis: theta rows per chunk
#define LG_SEG 32     // largest recurrence checkpoint spacing in k (== LG_BK)
#define LG_THREADS 256

// pipeline stages (for shtns_b200_stage_times)
#define SHTB_NSTAGES 6   // 0 prologue, 1 Legendre synthesis, 2 FFT synthesis, 3 FFT analysis, 4 Legendre analysis, 5 epilogue

#define FFT_MAX_FACTORS 16
#define FFT_NB 2      // butterflies held in registers per thread and pass

// Per-order metadata, one entry per im = 0..mmax (int arrays on the device).
struct MTables {
	int* koff;    // first row of order im in the k-major coefficient buffer
	int* coff;    // offset into the Ishioka recurrence coefficients (2 per k)
	int* xoff;    // offset into the Ishioka basis-change coefficients (3 per k)
	int* voff;    // offset into per-degree vector coefficients (degrees m..lmax+1)
	int* ckoff;   // first checkpoint segment of order im
	int* tm;      // first theta row (north index) kept by the polar threshold
};

// Public prefix must stay identical to shtns.h:struct shtns_info.
struct shtns_info {
	unsigned int nlm;
	unsigned short lmax;
	unsigned short mmax;
	unsigned short mres;
	unsigned short nlat_2;
	unsigned int nlat;
	unsigned int nphi;
	unsigned int nspat;
	unsigned short *li;
	unsigned short *mi;
	double *ct, *st;
	unsigned int nlat_padded;
	unsigned int nlm_cplx;
	// ---------------- private ----------------
	int norm_flags;          // shtns_norm | SHT_NO_CS_PHASE | SHT_REAL_NORM
	int base_norm;           // shtns_norm without flags
	int cs_phase;            // 1 with Condon-Shortley phase
	double mpos_renorm;      // 1.0 (complex convention) or 0.5 (SHT_REAL_NORM)
	int layout;              // layout bits given to shtns_set_grid
	int phi_contiguous;
	int south_first;
	int robert;
	int grid_set;
	double eps;
	int batch;               // fields per transform
	long spec_dist, spat_dist;
	// host tables
	std::vector<unsigned short> li_v, mi_v;
	std::vector<double> ct_v, st_v;      // full grid (public ct/st point here)
	std::vector<double> wq;              // Gauss weights of the north rows (sum over both hemispheres = 2)
	std::vector<double> alm;             // classic recurrence: per m pairs, reference layout (sht_legendre.c:630-657)
	std::vector<long> alm_off;           // offset of order im in alm
	std::vector<double> ish_c;           // Ishioka recurrence coefficients (2 per k)
	std::vector<double> ish_xs, ish_xa;  // Ishioka basis change for synthesis / analysis (3 per k)
	std::vector<double> stdt_lo, stdt_hi, van_lo, van_hi;   // per degree l = m..lmax+1
	std::vector<double> l_2;             // 1/(l(l+1)), l_2[0] = 0
	std::vector<int> koff_h, coff_h, xoff_h, voff_h, ckoff_h, tm_h, kmax_h;
	long ktot, ctot, xtot, vtot, segtot;
	int ckseg;                           // checkpoint spacing in k
	int fft_pairs;                       // latitude pairs per FFT CTA (0: automatic)
	int fft_generic;                     // FFT kernels: 0 automatic, 1 generic mixed-radix, 2 fused without prefetch, 3 no tensor stores
	int fft_extra_tx;                    // test hook: bytes the prefetching FFT kernels expect beyond their copies (0)
	int tile_wm;                         // Legendre tile shape option (0 automatic)
	std::vector<int> fft_radix;          // factorisation of nphi
	double Y00_1, Y10_ct, Y11_st;
	// device tables
	int dev;
	double *d_x, *d_x2, *d_s, *d_sinv, *d_w;   // north rows: |cos|, cos^2, sin, 1/sin, analysis weights
	double *d_c, *d_xs, *d_xa;
	double *d_stdt_lo, *d_stdt_hi, *d_van_lo, *d_van_hi, *d_l2;
	double2 *d_ck;                      // checkpoints (Y_k, Y_k+1), [segment][north row]
	double2 *d_tw;                       // exp(+2 pi i j / nphi), j < nphi
	double2 *d_tw4;                      // nphi = 12288: four-step factor tables (96 + 128 entries)
	double *d_fscr; size_t fscr_cap;     // four-step FFT analysis scratch (grow on demand)
	MTables mt;
	int *d_mint;                         // backing store of mt
	size_t table_bytes;
	// work buffers (grow on demand)
	double *d_qq; size_t qq_cap;         // k-major coefficient buffer [row][col]
	double2 *d_F; size_t F_cap;          // Fourier coefficients [fc][im][theta]
	void *d_stage; size_t stage_cap;     // device staging for host-pointer transforms
	// split-precision synthesis (shtns_b200_set_option 4): slices per operand
	// (0 = FP64 contraction) and its tables and buffers, allocated on first use
	// and owned by each plan object (clones included)
	int split_ns;
	short *d_yexp;                       // row exponents [im][north row]
	int *d_boff;                         // first 64-step chunk of each order in d_bsl
	long split_chunks;                   // chunks over all orders
	int split_kc;                        // steps per chunk of d_boff
	void *d_bsl; size_t bsl_cap;         // coefficient slices
	int *d_bexp; size_t bexp_cap;        // column exponents [im][column]
	int *d_split_err;                    // set by the kernel when a wait gives up
	// split precision from a precomputed digit table (option 4 with option 8 = 0):
	// Y_k(theta) of every order as int8 digits, built on first use and owned by
	// the original plan (clones use their base plan's table)
	int split_form;                      // 0 digit table (synthesis and analysis), 1 on-the-fly FP16 (synthesis only)
	void *d_ptab; size_t ptab_bytes;     // digit table
	int ptab_ns;                         // digits per value of the table
	long *d_ptoff;                       // per order: first 16 KB digit-block of the order
	long *d_pkoff;                       // per order: first 128-step block (coefficient digit stacks)
	long *d_pvoff;                       // per order: first kept theta tile (weighted Fourier digit stacks)
	int *d_pt0;                          // per order: first theta tile kept by the polar threshold
	int *d_pkf;                          // per (order, kept theta tile): first step block with a nonzero digit
	long ptab_kblocks, ptab_ttiles;      // sums over the orders of the above counts
	std::vector<long> koff_blocks_h;     // host copy of d_pkoff
	void *d_pbs; size_t pbs_cap;         // per call: B-operand digit stacks
	int *d_pexp; size_t pexp_cap;        // per call: column exponents [im][column]
	// FP64 Legendre values from a precomputed table (option 10): Y_k(theta) of
	// every order in 32 x 32 blocks, built on first use and owned by the
	// original plan (clones use their base plan's table)
	int ftab_mode;                       // 0 automatic (within a memory budget), 1 off, 2 on
	double *d_ftab; size_t ftab_bytes;   // table blocks
	long *d_ftoff;                       // per order: first block
	int *d_ftb0;                         // per order: first 32-latitude block kept by the polar threshold
	double *d_fzero;                     // one zero row of the B operand (steps beyond the call's last)
	int ftab_failed;                     // the automatic mode could not allocate the table: do not retry
	// local evaluation (points, latitudes, operators): classic-recurrence
	// tables on the device, allocated on first use (no grid needed), and staging
	double *d_alm; long *d_almoff;
	void *d_loc; size_t loc_cap;
	cudaStream_t comp_stream, xfer_stream;
	cudaStream_t d2h_stream;             // host-pointer transforms: device->host copies (created on first use)
	std::vector<cudaEvent_t> xev;        // host-pointer transforms: chunk events (created on first use)
	int own_xfer;
	int is_clone;
	shtns_cfg base;                      // plan whose tables a clone shares (NULL for originals)
	int nclones;
	// optional per-stage timing with CUDA events on the compute stream
	int timing;
	std::vector<cudaEvent_t> ev;         // pool: pairs (start, stop)
	std::vector<int> ev_stage;           // stage of each used pair
	int ev_used;
	double stage_ms[SHTB_NSTAGES];
	long stage_calls[SHTB_NSTAGES];
};

// ---- kernel parameter blocks ----
// Fourier rows split over several buffers by blocks of grid rows (the
// order-split transform with its exchange fused into the Legendre kernels):
// block b holds rows lat0[b] .. lat0[b+1]-1 as [fc][im][row - lat0[b]] with
// mstride orders per field-component.  n = 0: the plain buffer F.
#define SHTB_MAX_BLOCKS 16
struct RowBlocks {
	int n;
	int mstride;
	int lat0[SHTB_MAX_BLOCKS + 1];
	double2* base[SHTB_MAX_BLOCKS];
};

struct LegParams {
	int nlat, nlat_2, llim, mlim, mres, vec_extra;
	int im0;                             // first order of the launch (orders im0..mlim; 0 for whole transforms)
	int ncol, nfc;
	int ckseg;                           // checkpoint spacing in k (8, 16 or 32)
	int tile_wm;                         // Legendre tile: warps along the rows (1, 2, 4; 0 automatic)
	int south_first, robert;
	double mpos_inv;                     // analysis factor for m>0 (1/mpos_renorm)
	int adjoint;                         // 1: adjoint transforms (see sht_api.cu)
	double nphi;                         // longitudes (adjoint scalings)
	const double *x, *x2, *sinv, *w, *c;
	const double2 *ck;
	MTables mt;
	int nf;                              // fields per component (fc = component * nf + field)
	int ctype[3];                        // per component: 0 scalar, 1 V, 2 W
	double *qq;                          // coefficient buffer
	double2 *F;                          // Fourier buffer
	long fstride;                        // complex elements between field-components in F
	RowBlocks rb;                        // rows in per-block buffers instead of F (rb.n > 0)
};

// address of Fourier row `row` of field-component fc, order im (the
// tensor-core tiles are compiled separately for the block-split layout, so
// that the plain one keeps its registers)
__device__ __forceinline__ double2* fourier_row(const LegParams& p, int fc, int im, int row)
{
	if (p.rb.n == 0) return p.F + (long)fc * p.fstride + (long)im * p.nlat + row;
	int b = 0;
	while (b + 1 < p.rb.n && row >= p.rb.lat0[b + 1]) b++;
	const int r0 = p.rb.lat0[b];
	return p.rb.base[b] + ((long)fc * p.rb.mstride + im) * (p.rb.lat0[b + 1] - r0) + (row - r0);
}

struct PrepParams {
	int lmax, llim, mlim, mres, nf, ncomp, ncol, comp_type[3];   // comp_type: 0 scalar Q, 1 V (from S,T), 2 W (from S,T)
	int im0;                             // first order of the launch (0 for whole transforms)
	int msign;                           // -1: order -m in the vector terms (negative im of the _ml transforms)
	int neg_from;                        // > 0: fields f >= neg_from use -m in the vector terms (complex-field transforms)
	const double2 *Q, *S, *T;            // spectral inputs (may be null: zeros)
	double2 *Qo, *So, *To;               // spectral outputs (analysis)
	long spec_dist;
	const double *xs, *xa, *stdt_lo, *stdt_hi, *van_lo, *van_hi, *l2;
	MTables mt;
	double *qq;
};

struct FftParams {
	int N, S, nlat, mlim, nradix;
	unsigned long long rcode;            // radices of nphi, 4 bits each, first pass in the low bits
	const double2 *tw;
	double2 *F;
	long fstride;                        // complex elements between field-components in F
	double *spat[3];                     // per component base pointer
	const double *spat_in[3];
	int nf;                              // fields per component
	long spat_dist;
	int phi_contiguous;
	int vec2;                            // spatial pointers 16-byte aligned: latitude pairs moved as double2
	int extra_tx;                        // test hook: extra bytes expected per prefetched tile (0)
	int generic;                         // 0 automatic, 1 generic mixed-radix kernels, 2 fused kernels without prefetch,
	                                     // 3 prefetched loads with per-thread stores
	const double2 *tw1, *tw2;            // four-step FFT (nphi = 96 x 128): exp(+2 pi i j / 96), exp(+2 pi i j / 128)
	double *scratch;                     // four-step analysis: a grid per field-component (null: other kernels)
};

// ---- one transform call: its shape and the kernels' parameter blocks (sht_api.cu) ----
struct Job {
	int ncomp;
	int type[3];      // 0 scalar, 1 V (theta / spheroidal), 2 W (phi / toroidal)
	int nf, nfc, ncol, llim, mlim, vec_extra;
};
// Fills j for ncomp components of the given types at truncation ltr and grows
// the plan's work buffers named by bufs (1 coefficient buffer, 2 Fourier
// buffer; 0 allocates nothing).  false (error recorded) on a bad call.
bool setup_job(shtns_cfg s, Job& j, int ncomp, const int* types, int ltr, unsigned bufs = 3);
// Parameter blocks with every plan option applied; work-buffer pointers are
// the plan's own (d_qq, d_F), which a caller may replace.
LegParams leg_params(shtns_cfg s, const Job& j);
PrepParams prep_params(shtns_cfg s, const Job& j);
FftParams fft_params(shtns_cfg s, const Job& j, int nrows = 0);

// ---- launchers (sht_legendre.cu / sht_fft.cu) ----
void launch_checkpoints(shtns_cfg s, cudaStream_t st);
void launch_prep_synth(const PrepParams& p, cudaStream_t st);
void launch_post_analys_m(const PrepParams& p, int mmax, cudaStream_t st);
void launch_leg_synth(const LegParams& p, cudaStream_t st);
void launch_leg_analys(const LegParams& p, int kmax_all, cudaStream_t st);
void launch_leg_synth_split(shtns_cfg s, const LegParams& p, cudaStream_t st);
bool split_row_exponents(shtns_cfg s, cudaStream_t st);
void launch_ptab_synth(shtns_cfg s, const LegParams& p, cudaStream_t st);
void launch_ptab_analys(shtns_cfg s, const LegParams& p, cudaStream_t st);
void free_ptab(shtns_cfg s);
bool launch_ftab_synth(shtns_cfg s, const LegParams& p, cudaStream_t st);
void free_ftab(shtns_cfg s);
bool leg_simt_selected(const LegParams& p, bool synth);
void launch_leg_synth_simt(const LegParams& p, cudaStream_t st);
void launch_leg_analys_simt(const LegParams& p, int kmax_all, cudaStream_t st);
void free_split(shtns_cfg s);
void launch_leg_multi(const LegParams* d_plist, const int4* d_work, int nwork, int* d_counter, int ckseg, bool synth,
                      int nctas, cudaStream_t st);
int fft_threads(int N, int S, unsigned long long rcode, int nradix);
bool fft_fused_available(int N);
size_t fft_smem_bytes(int N, int S);
void launch_fft_synth(const FftParams& p, int nfc, cudaStream_t st);
void launch_fft_analys(const FftParams& p, int nfc, cudaStream_t st);
int fft_take_wait_error();
int fft_last_path();

// ---- Gauss-Legendre grid on the current device (sht_gauss.cu) ----
bool gauss_grid_gpu(int n, std::vector<double>& x, std::vector<double>& st, std::vector<double>& w);

// ---- static scratch of cu_SH_to_spat_noalloc (sht_noalloc.cu) ----
int shtb_noalloc_fill(int byte);

// ---- error reporting (sht_plan.cu) ----
void shtb_set_error(int code, const std::string& msg);
void shtb_count_launch(int n = 1);
bool shtb_cuda_ok(cudaError_t e, const char* where);
void shtb_stage_begin(shtns_cfg s, int stage);
void shtb_stage_end(shtns_cfg s);
void shtb_timing_release(shtns_cfg s);
extern "C" int shtns_b200_set_option(shtns_cfg s, int option, int value);
