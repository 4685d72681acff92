/*
 * shtns.h -- public C API of shtns_b200, a drop-in replacement for the
 * SHTns 3.5.2 transform API whose transforms run on an NVIDIA B200 (sm_100a).
 *
 * Every declaration below keeps the name, signature, argument meaning and
 * return value of the SHTns 3.5.2 function it replaces (the reference
 * shtns.h line is given beside each), so code written against SHTns compiles
 * and links against libshtns_b200.so unchanged.  Host-pointer transforms
 * (SH_to_spat, ...) copy their arrays to the GPU, transform there and copy
 * back; the cu_* functions of shtns_cuda.h take device pointers.
 *
 * Local evaluation (points, one latitude), Legendre arrays, the l+-1
 * operators and rotations run on the GPU as well (host arrays are copied in
 * and out).  Regular (non-Gauss) grids are not provided.
 */
#ifndef SHTNS_B200_SHTNS_H
#define SHTNS_B200_SHTNS_H

#include <stddef.h>

#ifdef __cplusplus
	#include <complex>
	typedef std::complex<double> cplx;
	typedef std::complex<float> cplx_f;
#else
	#include <complex.h>
	typedef complex double cplx;
	typedef complex float cplx_f;
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* interface version: same encoding as the reference (shtns.h:39) */
#define SHTNS_INTERFACE 0x30500

/* plan handle (shtns.h:42) */
typedef struct shtns_info* shtns_cfg;

/* rotation handle (shtns.h:43-44) */
typedef struct shtns_rot_* shtns_rot;

/* normalisations (shtns.h:48-55) */
enum shtns_norm {
	sht_orthonormal,
	sht_fourpi,
	sht_schmidt,
	sht_for_rotations
};
#define SHT_NO_CS_PHASE (256*4)
#define SHT_REAL_NORM (256*8)

/* grid types and layout flags (shtns.h:58-75).  Only Gauss grids are
 * provided: sht_gauss, sht_auto, sht_quick_init and sht_gauss_fly. */
enum shtns_type {
	sht_gauss,
	sht_auto,
	sht_reg_fast,
	sht_reg_dct,
	sht_quick_init,
	sht_reg_poles,
	sht_gauss_fly
};
#define SHT_NATIVE_LAYOUT 0
#define SHT_THETA_CONTIGUOUS 256
#define SHT_PHI_CONTIGUOUS (256*2)
#define SHT_SOUTH_POLE_FIRST (256*32)
#define SHT_SCALAR_ONLY (256*16)
#define SHT_LOAD_SAVE_CFG (256*64)
#define SHT_ALLOW_GPU (256*128)
#define SHT_ALLOW_PADDING (256*256)

#ifndef SHTNS_B200_PRIVATE
/* read-only public part of the plan, layout-compatible with shtns.h:79-94 */
struct shtns_info {
	const unsigned int nlm;
	const unsigned short lmax;
	const unsigned short mmax;
	const unsigned short mres;
	const unsigned short nlat_2;
	const unsigned int nlat;
	const unsigned int nphi;
	const unsigned int nspat;
	const unsigned short *const li;
	const unsigned short *const mi;
	const double *const ct;
	const double *const st;
	const unsigned int nlat_padded;
	const unsigned int nlm_cplx;
};
#endif

/* index macros (shtns.h:104-106) */
#define LiM(shtns, l,im) ( (((im)*(2*shtns->lmax + 2 - ((im)+1)*shtns->mres))>>1) + (l) )
#define LM(shtns, l,m) ( (((((unsigned short)(m))/shtns->mres)*(2*shtns->lmax + 2 - ((m)+shtns->mres)))>>1) + (l) )
#define LM_LOOP( shtns, action ) { int lm=0; do { action } while(++lm < shtns->nlm); }
#define LM_L_LOOP( shtns, action ) { int lm=0; do { int l=shtns->li[lm]; action } while(++lm < shtns->nlm); }
#define NSPAT_ALLOC(shtns) (shtns->nspat)
#define PHI_DEG(shtns, ip) (360./(shtns->nphi*shtns->mres))*(ip)
#define PHI_RAD(shtns, ip) (2.*M_PI/(shtns->nphi*shtns->mres))*(ip)

long nlm_calc(long lmax, long mmax, long mres);                 /* shtns.h:133 */
long nlm_cplx_calc(long lmax, long mmax, long mres);            /* shtns.h:136 */
void shtns_verbose(int);                                        /* shtns.h:138 */
void shtns_print_version(void);                                 /* shtns.h:139 */
const char* shtns_get_build_info(void);                         /* shtns.h:140 */
void shtns_print_cfg(shtns_cfg);                                /* shtns.h:144 */

shtns_cfg shtns_init(enum shtns_type flags, int lmax, int mmax, int mres, int nlat, int nphi);   /* shtns.h:149 */
shtns_cfg shtns_create(int lmax, int mmax, int mres, enum shtns_norm norm);                     /* shtns.h:151 */
int shtns_set_grid(shtns_cfg, enum shtns_type flags, double eps, int nlat, int nphi);           /* shtns.h:153 */
int shtns_set_grid_auto(shtns_cfg, enum shtns_type flags, double eps, int nl_order, int *nlat, int *nphi); /* shtns.h:155 */
shtns_cfg shtns_create_with_grid(shtns_cfg, int mmax, int nofft);                                /* shtns.h:157 */
int shtns_use_threads(int num_threads);                         /* shtns.h:159 */
int shtns_use_gpu(int device_id);                               /* shtns.h:161 */
void shtns_reset(void);                                         /* shtns.h:163 */
void shtns_destroy(shtns_cfg);                                  /* shtns.h:164 */
void shtns_unset_grid(shtns_cfg);                               /* shtns.h:165 */
void shtns_robert_form(shtns_cfg, int robert);                  /* shtns.h:168 */
void* shtns_malloc(size_t bytes);                               /* shtns.h:170 */
void shtns_free(void* p);                                       /* shtns.h:171 */

double sh00_1(shtns_cfg);                                       /* shtns.h:178 */
double sh10_ct(shtns_cfg);                                      /* shtns.h:179 */
double sh11_st(shtns_cfg);                                      /* shtns.h:180 */
double shlm_e1(shtns_cfg, int l, int m);                        /* shtns.h:181 */
int shtns_gauss_wts(shtns_cfg, double *wts);                    /* shtns.h:183 */

/* scalar transforms (shtns.h:262-267); spat_to_SH leaves Vr unchanged */
void spat_to_SH(shtns_cfg shtns, double *Vr, cplx *Qlm);
void SH_to_spat(shtns_cfg shtns, cplx *Qlm, double *Vr);
/* 2-D vector transforms (shtns.h:282-288) */
void spat_to_SHsphtor(shtns_cfg, double *Vt, double *Vp, cplx *Slm, cplx *Tlm);
void SHsphtor_to_spat(shtns_cfg, cplx *Slm, cplx *Tlm, double *Vt, double *Vp);
void SHsph_to_spat(shtns_cfg, cplx *Slm, double *Vt, double *Vp);
void SHtor_to_spat(shtns_cfg, cplx *Tlm, double *Vt, double *Vp);
#define SH_to_grad_spat(shtns, S,Gt,Gp) SHsph_to_spat(shtns, S, Gt, Gp)
/* 3-D vector transforms (shtns.h:303-306) */
void spat_to_SHqst(shtns_cfg, double *Vr, double *Vt, double *Vp, cplx *Qlm, cplx *Slm, cplx *Tlm);
void SHqst_to_spat(shtns_cfg, cplx *Qlm, cplx *Slm, cplx *Tlm, double *Vr, double *Vt, double *Vp);
/* truncated transforms (shtns.h:315-324) */
/* Complex-valued fields, mres = 1 (shtns.h:268-309): alm[LM_cplx(l, m)],
 * -l <= m <= l, nlm_cplx coefficients; complex spatial arrays of nspat */
void SH_to_spat_cplx(shtns_cfg, cplx *alm, cplx *z);                                               /* shtns.h:272 */
void spat_cplx_to_SH(shtns_cfg, cplx *z, cplx *alm);                                               /* shtns.h:277 */
void SHsphtor_to_spat_cplx(shtns_cfg, cplx *Slm, cplx *Tlm, cplx *Vt, cplx *Vp);                   /* shtns.h:294 */
void spat_cplx_to_SHsphtor(shtns_cfg, cplx *Vt, cplx *Vp, cplx *Slm, cplx *Tlm);                   /* shtns.h:292 */
void SHqst_to_spat_cplx(shtns_cfg, cplx *Qlm, cplx *Slm, cplx *Tlm, cplx *Vr, cplx *Vt, cplx *Vp); /* shtns.h:309 */
void spat_cplx_to_SHqst(shtns_cfg, cplx *Vr, cplx *Vt, cplx *Vp, cplx *Qlm, cplx *Slm, cplx *Tlm); /* shtns.h:308 */

/* Legendre transforms at one order m = |im|*mres, no FFT (shtns.h:329-342):
 * spectral lmax+1-m coefficients of that order, spatial nlat complex values */
void spat_to_SH_ml(shtns_cfg, int im, cplx *Vr, cplx *Ql, int ltr);                                  /* shtns.h:333 */
void SH_to_spat_ml(shtns_cfg, int im, cplx *Ql, cplx *Vr, int ltr);                                  /* shtns.h:334 */
void spat_to_SHsphtor_ml(shtns_cfg, int im, cplx *Vt, cplx *Vp, cplx *Sl, cplx *Tl, int ltr);        /* shtns.h:336 */
void SHsphtor_to_spat_ml(shtns_cfg, int im, cplx *Sl, cplx *Tl, cplx *Vt, cplx *Vp, int ltr);        /* shtns.h:337 */
void SHsph_to_spat_ml(shtns_cfg, int im, cplx *Sl, cplx *Vt, cplx *Vp, int ltr);                     /* shtns.h:338 */
void SHtor_to_spat_ml(shtns_cfg, int im, cplx *Tl, cplx *Vt, cplx *Vp, int ltr);                     /* shtns.h:339 */
void spat_to_SHqst_ml(shtns_cfg, int im, cplx *Vr, cplx *Vt, cplx *Vp, cplx *Ql, cplx *Sl, cplx *Tl, int ltr); /* shtns.h:341 */
void SHqst_to_spat_ml(shtns_cfg, int im, cplx *Ql, cplx *Sl, cplx *Tl, cplx *Vr, cplx *Vt, cplx *Vp, int ltr); /* shtns.h:342 */

void spat_to_SH_l(shtns_cfg, double *Vr, cplx *Qlm, int ltr);
void SH_to_spat_l(shtns_cfg, cplx *Qlm, double *Vr, int ltr);
void SHsphtor_to_spat_l(shtns_cfg, cplx *Slm, cplx *Tlm, double *Vt, double *Vp, int ltr);
void SHsph_to_spat_l(shtns_cfg, cplx *Slm, double *Vt, double *Vp, int ltr);
void SHtor_to_spat_l(shtns_cfg, cplx *Tlm, double *Vt, double *Vp, int ltr);
void spat_to_SHsphtor_l(shtns_cfg, double *Vt, double *Vp, cplx *Slm, cplx *Tlm, int ltr);
void spat_to_SHqst_l(shtns_cfg, double *Vr, double *Vt, double *Vp, cplx *Qlm, cplx *Slm, cplx *Tlm, int ltr);
void SHqst_to_spat_l(shtns_cfg, cplx *Qlm, cplx *Slm, cplx *Tlm, double *Vr, double *Vt, double *Vp, int ltr);
#define SH_to_grad_spat_l(shtns, S,Gt,Gp,ltr) SHsph_to_spat_l(shtns, S, Gt, Gp, ltr)

/* Local and partial evaluation (shtns.h:349-363); no grid needed.  Points
 * at cos(theta) = cost and longitude phi; latitudes on nphi equispaced
 * longitudes phi_j = 2 pi j / nphi, truncated at degree ltr and order mtr. */
double SH_to_point(shtns_cfg, cplx *Qlm, double cost, double phi);                                  /* shtns.h:352 */
cplx SH_to_point_cplx(shtns_cfg, cplx *alm, double cost, double phi);                                /* shtns.h:353 */
void SH_to_grad_point(shtns_cfg, cplx *DrSlm, cplx *Slm,
                      double cost, double phi, double *vr, double *vt, double *vp);                  /* shtns.h:354 */
void SHqst_to_point(shtns_cfg, cplx *Qlm, cplx *Slm, cplx *Tlm,
                    double cost, double phi, double *vr, double *vt, double *vp);                    /* shtns.h:356 */
void SH_to_lat(shtns_cfg shtns, cplx *Qlm, double cost, double *vr, int nphi, int ltr, int mtr);     /* shtns.h:359 */
void SHqst_to_lat(shtns_cfg, cplx *Qlm, cplx *Slm, cplx *Tlm, double cost,
                  double *vr, double *vt, double *vp, int nphi, int ltr, int mtr);                   /* shtns.h:361 */

/* Associated Legendre functions of order im*mres at x = cos(theta), degrees
 * m..lmax, normalised as the plan's harmonics (shtns.h:232-233); the _deriv
 * form returns P/sin(theta) (m > 0) and dP/dtheta.  Return the first degree
 * whose value is not negligible (values below are written as 0). */
int legendre_sphPlm_array(shtns_cfg shtns, const int lmax, const int im, const double x, double *yl); /* shtns.h:232 */
int legendre_sphPlm_deriv_array(shtns_cfg shtns, const int lmax, const int im, const double x,
                                const double sint, double *yl, double *dyl);                         /* shtns.h:233 */

/* Rotations (shtns.h:186-218).  SH_Zrotate rotates about the z axis by alpha
 * (Rlm = Qlm e^{-i m alpha}); SH_Yrotate, SH_Yrotate90 and SH_Xrotate90 need
 * mres = 1 and mmax = lmax.  Rotation objects take Euler angles (intrinsic
 * ZYZ or ZXZ) or an angle and an axis and apply the rotation to orthonormal
 * expansions of real (LM layout) or complex (LM_cplx layout) fields; Rlm may
 * be Qlm.  All rotations are active rotations of the field. */
void SH_Zrotate(shtns_cfg, cplx *Qlm, double alpha, cplx *Rlm);                                      /* shtns.h:192 */
void SH_Yrotate(shtns_cfg, cplx *Qlm, double alpha, cplx *Rlm);                                      /* shtns.h:194 */
void SH_Yrotate90(shtns_cfg, cplx *Qlm, cplx *Rlm);                                                  /* shtns.h:196 */
void SH_Xrotate90(shtns_cfg, cplx *Qlm, cplx *Rlm);                                                  /* shtns.h:198 */
shtns_rot shtns_rotation_create(const int lmax, const int mmax, int norm);                           /* shtns.h:202 */
void shtns_rotation_destroy(shtns_rot r);                                                            /* shtns.h:204 */
void shtns_rotation_set_angles_ZYZ(shtns_rot r, double alpha, double beta, double gamma);            /* shtns.h:206 */
void shtns_rotation_set_angles_ZXZ(shtns_rot r, double alpha, double beta, double gamma);            /* shtns.h:208 */
void shtns_rotation_set_angle_axis(shtns_rot r, double theta, double Vx, double Vy, double Vz);      /* shtns.h:210 */
int shtns_rotation_wigner_d_matrix(shtns_rot r, const int l, double *mx);                            /* shtns.h:214 */
void shtns_rotation_apply_cplx(shtns_rot r, cplx *Zlm, cplx *Rlm);                                   /* shtns.h:216 */
void shtns_rotation_apply_real(shtns_rot r, cplx *Qlm, cplx *Rlm);                                   /* shtns.h:218 */

/* Operators coupling degrees l-1 and l+1 (shtns.h:240-245):
 * Rlm[lm] = mx[2*lm] * Qlm[lm-1] + mx[2*lm+1] * Qlm[lm+1]; mx holds 2*nlm doubles. */
void mul_ct_matrix(shtns_cfg, double *mx);                                                           /* shtns.h:240 */
void st_dt_matrix(shtns_cfg, double *mx);                                                            /* shtns.h:243 */
void SH_mul_mx(shtns_cfg, double *mx, cplx *Qlm, cplx *Rlm);                                         /* shtns.h:245 */

#ifdef __cplusplus
}
#endif

#endif /* SHTNS_B200_SHTNS_H */
