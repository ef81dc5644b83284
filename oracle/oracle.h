/*
 * oracle.h -- ORACLE: CPU restatement of the reference Fortran hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (radtrancode_b200/)
 * links, loads or calls this code; only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg use it, as the checker.
 *
 * Parity status: the reference ships no golden vectors or tests for this
 * path and no Fortran compiler exists on these machines, so the restatement
 * is pinned by analytic known-answer tests, finite differences, invariants
 * and the real CIA table shipped with the reference (raddata/isotest.tab)
 * -- "parity unpinned" against the reference binary itself.
 *
 * Two precisions:
 *   ORC_MIXED (0): the reference's own REAL/DOUBLE PRECISION mix, including
 *                  sngl() casts, FP64 transmissions, FP64 cumulative g
 *                  weights; EXP(REAL) is the deterministic exponential of
 *                  detexp.h.  This mode is the bit-exactness yardstick for
 *                  the integer g-bin assignment.
 *   ORC_FP64  (1): every REAL promoted to DOUBLE; the accuracy yardstick.
 */
#ifndef RTB_ORACLE_H
#define RTB_ORACLE_H

#include <stdint.h>
#include "../include/radtran_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MIXED 0
#define ORC_FP64  1

typedef struct orc_tables {
    /* k-tables: same meaning and layout as rtb_set_ktables */
    int ntab, np, nt, ng;
    const float* lnp;
    const float* tk;
    const float* delg;
    const float* vmin;
    const float* delv;
    const int*   nbin;
    const float* data;
    /* CIA table: same meaning as rtb_set_cia; has_cia = 0 -> CIA off */
    int has_cia;
    float dnu;
    const double* cia_temps;
    const float* kcia;
    /* irregular wavenumber grids (delv <= 0, the same for every table): the
     * first table's centres VCEN(npoint) (read_klist.f:141-145); else NULL */
    int npoint;
    const float* vcen;
    /* para-H2 CIA (fpread_all): same meaning as rtb_set_para_cia; has_para = 0 -> none */
    int has_para, ipara;
    float dnu2;
    const float* para_temps;
    const float* para_fp;
    const float* kh2h2;
    const float* kh2he;
    const float* kcia5;
    /* e3interp's table (IMOD 18): 1001 transmissions and E3; NULL -> none */
    const double* e3_tran;
    const double* e3_e3;
    /* /solardat/ of init_solar_wave (iform 1, 4): npt = 0 -> none */
    int solar_npt;
    const float* solar_wave;
    const float* solar_rad;
} orc_tables;

/* Debug capture of the g-bin assignment (mixed mode), one record per
 * (wavenumber, layer, overlap pass igas = 1..ngas-1):
 *   perm [(iw*nlayer + il)*(ngas-1) + (igas-1)][ng*ng]  sorted element ids
 *   split[(iw*nlayer + il)*(ngas-1) + (igas-1)][ng]      sorted position of the
 *        element at which bin b is closed (rankg.f:118-141), -1 if none.
 * Passes that do not sort (a zero distribution, noverlapg.f:88-108) hold -1.
 * ties[(iw*nlayer + il)*(ngas-1) + (igas-1)] counts adjacent equal sorted
 * keys (heapsort order of tied keys is what fixes their bin).
 * Any pointer may be NULL. */
typedef struct orc_debug {
    int16_t* perm;
    int16_t* split;
    int16_t* ties;   /* [...] number of adjacent equal keys after the sort */
} orc_debug;

/* cirsrtfg_wave restatement (radtran/cirsradg/cirsrtfg_wave.f:290-516)
 * Outputs (double, packed as rtb_cirsrtfg_wave): calcout, gradients,
 * gradtsurf (may be NULL).  Returns RTB_* status. */
int orc_cirsrtfg_wave(const orc_tables* tab, const rtb_atm* atm, int precision,
                      double* calcout, double* gradients, double* gradtsurf,
                      const orc_debug* dbg);

/* Same, running independent wavenumbers on `nthreads` host threads (the
 * reference loop over wavenumbers has no carried state); dbg (may be NULL)
 * as above, each thread writing the records of its own wavenumbers. */
int orc_cirsrtfg_wave_mt(const orc_tables* tab, const rtb_atm* atm, int precision,
                         double* calcout, double* gradients, double* gradtsurf,
                         int nthreads, const orc_debug* dbg);

/* --- unit-level entry points used by the oracle's own tests ----------- */
/* 0 = reference heapsort (default); 1 = stable sort (tie-order experiments) */
void  orc_set_sort_mode(int mode);
float orc_det_expf_c(float x);
/* locate.f (radtran/scatter/locate.f:1-28), 1-based result */
int   orc_locate(const float* xx, int n, float x);
/* sort2g.f heapsort: sorts ra[0..n-1] ascending in place and returns the
 * 0-based permutation in ib */
void  orc_sort2g(int n, float* ra, int* ib);
/* rankg.f on one set of combined elements (mixed precision). grad is
 * [nparam][nloop] (column per parameter); outputs k_g[ng], dkdq[nparam][ng],
 * perm[nloop], split[ng].  Returns 0 or RTB_ERR_GORD. */
int   orc_rankg(int nparam, const float* gw, int ng, int nloop,
                const float* weight, const float* cont, const float* grad,
                float* k_g, float* dkdq, int16_t* perm, int16_t* split);
/* planck_wave.f / planckg_wave.f (mixed) */
float orc_planck_wave(int ispace, float v, float t);
float orc_planckg_wave(int ispace, float v, float t);

/* --- Newton step (nemesis/calc_gain_matrix.f, calcnextxn.f,
 *     calc_phiret.f, radtran/matrices/dinvertm.f) ---------------------
 * Dense column-major arrays with leading dimensions ldy >= ny, ldx >= nx:
 *   kk (ldy, nx) REAL, sx (ldx, nx) REAL, sxi (ldx, nx) DOUBLE,
 *   se (ldy, ny) REAL, sei (ldy, ny) DOUBLE, dd (ldx, ny) DOUBLE,
 *   aa (ldx, nx) DOUBLE.  *icheck receives dinvertm's ICHECK. */
int orc_calc_gain_matrix(int nx, int ny, int ldx, int ldy,
                         const float* kk, const float* sx, const double* sxi,
                         const float* se, const double* sei,
                         double* dd, double* aa, int* icheck);
/* Diagonal-Se fast form of the nx<ny branch with the same FP64 Cholesky
 * inverse (mathematically identical; used to keep CPU baselines bounded). */
int orc_calc_gain_matrix_diag(int nx, int ny, int ldx, int ldy,
                              const float* kk, const double* sxi,
                              const double* sei_diag,
                              double* dd, double* aa, int* icheck);
void orc_calcnextxn(int nx, int ny, int ldx, const float* x0, const float* xn,
                    const float* y, const float* yn, const double* dd,
                    const double* aa, float* x_out);
float orc_calc_phiret(int ny, int ldy, const float* y, const float* yn,
                      const double* sei, int nx, int ldx, const float* xn,
                      const float* xa, const double* sai, float* chisq);
float orc_calc_phiret_diag(int ny, const float* y, const float* yn,
                           const double* sei_diag, int nx, int ldx,
                           const float* xn, const float* xa, const double* sai,
                           float* chisq);
/* calc_serr.f with a diagonal se (REAL se_diag[ny]); outputs REAL (ldx, nx) */
void orc_calc_serr_diag(int nx, int ny, int ldx, const float* sx_in, const float* se_diag, const double* dd_in,
                        const double* aa_in, float* st_out, float* sn_out, float* sm_out);
/* cirsconv.f for FWHM >= 0 (FWHM > 0: natural cubic spline, 20-point
 * trapezoid per channel; FWHM = 0: copy) */
int orc_cirsconv(int nwave, const float* vwave, const float* y, float fwhm, int nconv, const float* vconv,
                 float* yout);
/* cirsconv.f:12-246 in full: FWHM > 0 with an optional width table
 * (vfwhm, xfwhm; nfwhm = 0 for none), FWHM = 0, FWHM < 0 with nfil filter
 * functions (filter k: vcen[k], nsub[k] points of vfil/fil, concatenated),
 * nwave = 1 with FWHM != 0 */
int orc_cirsconv_ex(float fwhm, int nwave, const float* vwave, const float* y, int nconv, const float* vconv,
                    int nfwhm, const float* vfwhm, const float* xfwhm, int nfil, const float* vcen, const int* nsub,
                    const float* vfil, const float* fil, float* yout);
/* dinvertm(jmod=2): Cholesky inverse with the A*Ainv check; returns icheck */
int orc_dinvertm_chol(int n, int lda, const double* a, double* ainv);

/* --- retrieval loop (nemesis/coreret.f:520-1106) for the layer-state
 *     model of rtb_retrieve_batch ------------------------------------- */
#define ORC_TRACE_MAX 64
typedef struct orc_retrieval_trace {
    int n;                          /* iterations recorded */
    float phi[ORC_TRACE_MAX];       /* cost of the trial state (0: rejected before the forward model) */
    int verdict[ORC_TRACE_MAX];     /* 0 rejected before the forward model, 1 accepted, 2 rejected */
    float alambda[ORC_TRACE_MAX];   /* brake after the iteration */
} orc_retrieval_trace;
/* spectrum yn[ny] and kk[nx][ny] (gradients packing) at state x */
int orc_forward_state(const orc_tables* tab, const rtb_retrieval_spec* s, const float* x, int precision,
                      int nthreads, float* yn, float* kk);
int orc_retrieve(const orc_tables* tab, const rtb_retrieval_spec* s, const rtb_retrieval_opts* o, int precision,
                 int nthreads, rtb_retrieval_result* res, orc_retrieval_trace* tr);

/* LAYERG (radtran/path/layerg.f:146-458) and the nadir thermal path of ATMG
 * (radtran/path/atmg.f:250-373): the same arguments and outputs as
 * rtb_layerg, in REAL arithmetic */
int orc_layerg(const rtb_profile* prof, const rtb_layer_opts* opts, rtb_layers* out);

#ifdef __cplusplus
}
#endif
#endif
