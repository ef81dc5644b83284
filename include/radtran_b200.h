/*
 * radtran_b200.h -- C ABI of the B200-native CIRSRADG forward model with
 * analytic Jacobian and of the optimal-estimation Newton step.
 *
 * Every array argument is a plain host pointer laid out exactly as the
 * reference Fortran declares it (column-major, with the leading dimension
 * passed explicitly so that a Fortran caller can hand over its COMMON-block
 * arrays, dimensioned with MAXLAY/MAXPAT/MAXV/..., without repacking).
 * No torch or CUDA type appears in any signature.  Every entry point returns
 * an int status (RTB_OK == 0) instead of the reference's STOP; the message of
 * the last failure is available from rtb_last_error().
 *
 * Threading: one rtb_context is used by one host thread at a time (the
 * reference itself is not re-entrant: COMMON blocks, SAVEd read-once flags).
 * Several contexts may coexist, one per host thread.
 */
#ifndef RADTRAN_B200_H
#define RADTRAN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------- */
/* status codes                                                            */
/* ---------------------------------------------------------------------- */
#define RTB_OK              0
#define RTB_ERR_ARG         1   /* bad argument (NULL, negative size, ...) */
#define RTB_ERR_LIMIT       2   /* a MAX* limit is exceeded: check_limits.f STOPs here */
#define RTB_ERR_UNSUPPORTED 3   /* option outside the implemented path (IMOD 15, ILBL, ...) */
#define RTB_ERR_CUDA        4   /* CUDA runtime failure; the message names the call */
#define RTB_ERR_NOTABLE     5   /* no k-table / CIA table loaded in the context */
#define RTB_ERR_NONPD       6   /* Cholesky met a non-positive pivot (dcholdc.f:69-84) */
#define RTB_ERR_RANGE       7   /* a value is outside a table range where the reference STOPs */
#define RTB_ERR_GORD        8   /* g-ordinate walk ran past NG (rankg.f:147, uninitialised g_ord) */
#define RTB_ERR_BUDGET      9   /* request larger than the device memory budget */

/* Fortran parameters of the reference (radtran/includes/arrdef.f:18-22,
 * nemesis/arraylen.f:22); used as the default leading dimensions. */
#define RTB_MAXLAY  400
#define RTB_MAXPAT  200
#define RTB_MAXGAS  30
#define RTB_MAXCON  10
#define RTB_MAXG    51
#define RTB_MAXK    30
#define RTB_MAXV    401
#define RTB_MAXPRO  200
#define RTB_MY      2048
#define RTB_MX      401

/* CIA table shape (radtran/includes/ciacom.f:2-6) */
#define RTB_CIA_NUMPAIRS 9
#define RTB_CIA_NUMT     25
#define RTB_CIA_NUMWN    1501

typedef struct rtb_context rtb_context;

/* Create a context on CUDA device `device`.  Fails with RTB_ERR_CUDA when no
 * device is usable: there is no CPU fallback. */
int  rtb_create(int device, rtb_context** out);
void rtb_destroy(rtb_context* ctx);
const char* rtb_last_error(const rtb_context* ctx);
const char* rtb_version(void);

/* ---------------------------------------------------------------------- */
/* Resident tables                                                         */
/* ---------------------------------------------------------------------- */

/* Load the k-tables of a run into device memory once.
 * Replaces read_klist (radtran/cirsrad/read_klist.f:30) + read_khead
 * (radtran/cirsrad/read_khead.f:18) residency and the per-record direct-access
 * READs of get_kg (radtran/cirsradg/get_kg.f:228-304).
 *   ntab            number of tables (one per gas that has a .kta file)
 *   np, nt, ng      table grid (all tables share it, as the /INTERPK/ COMMON
 *                   block of get_kg.f:100-101 does); nt < 0 selects one
 *                   temperature grid of |nt| points per pressure (TEMP2)
 *   lnp[np]         log of the table pressures in atm (read_khead.f:81-84)
 *   tk              table temperatures, K: TEMP(nt), or for nt < 0
 *                   TEMP2(np, |nt|) column-major (pressure fastest)
 *   delg[ng]        g-ordinate weights (DEL_G)
 *   vmin[ntab], delv[ntab], nbin[ntab]   wavenumber grid of each table
 *                   (delv > 0: regular grid as in get_kg.f:193-208; delv <= 0:
 *                   an irregular grid, the same delv for every table, with
 *                   the centres given by rtb_set_ktable_centres)
 *   data            concatenation over tables of REAL k(ng, |nt|, np, nbin) in
 *                   record order: record = ((ibin*np + ip)*nt + it)*ng + ig,
 *                   i.e. exactly the .kta record order after IREC0, values
 *                   multiplied by 1e20 as stored in the files.
 * Tables stay resident until the next call or rtb_destroy. */
int rtb_set_ktables(rtb_context* ctx, int ntab, int np, int nt, int ng,
                    const float* lnp, const float* tk, const float* delg,
                    const float* vmin, const float* delv, const int* nbin,
                    const float* data);

/* The gas and isotope ids of the loaded tables (the .kta header's IDGAS,
 * ISOGAS; rtb_load_ktables sets them).  With them a gas's ktab may be
 * RTB_KTAB_BY_ID: its tables are every table of its ids, in load order, and
 * each calculation wavenumber takes the first regular table whose range
 * covers it (FINDLOC, read_klist.f:247-265) -- or, on an irregular grid, the
 * last of them (read_klist.f:266-310); a wavenumber no table covers gives
 * the gas zero k (lun = -99, read_klist.f:341-351).  Cleared by
 * rtb_set_ktables. */
#define RTB_KTAB_BY_ID (-2)
int rtb_set_ktable_ids(rtb_context* ctx, int ntab, const int* idgas, const int* isogas);

/* The centres VCEN(npoint) of irregular k-tables (delv <= 0; read_khead.f:
 * 100-103), those of the first table as read_klist.f:141-145 keeps them
 * (npoint = its nbin).  A calculation wavenumber takes the centre nearest in
 * per cent (delv < 0, coincident) or the nearest at or below it, weighted
 * with the next by FRACK (delv = 0), read_klist.f:266-310.  Cleared by
 * rtb_set_ktables. */
int rtb_set_ktable_centres(rtb_context* ctx, int npoint, const float* vcen);

/* Load a CIA table: replaces the one-time read of ciaread
 * (radtran/radtran/ciaread.f:63-105) into /CIATABLE/.
 *   dnu          wavenumber step of the table grid vvk1(i) = (i-1)*dnu
 *   temps[25]    DOUBLE temperatures as in the file's first record
 *   kcia         REAL kcia(9, 25, 1501), Fortran order (pair fastest). */
int rtb_set_cia(rtb_context* ctx, float dnu, const double* temps, const float* kcia);

/* Load the para-H2 CIA table of fpread_all (radtran/radtran/fpread_all.f,
 * the /FPTABLE/ block of ciacom.f), used instead of the CIA table for an
 * atmosphere with flagh2p = 1 (cirsradg_wave.f:634-640 calls NPARACON_ALL):
 *   dnu2           wavenumber step of the grid vvk2(i) = (i-1)*dnu2
 *   ipara          number of tabulated para-H2 fractions (12 or 24)
 *   temps[25]      REAL temperatures
 *   fp[ipara]      para-H2 fractions (nparacon_all.f assumes fp(1) = 0.25 and
 *                  an even spacing fp(2) - fp(1))
 *   kh2h2, kh2he   REAL (ipara, 25, 1501), Fortran order: H2-H2 and H2-He
 *   kcia5          REAL (5, 25, 1501): H2-N2, N2-CH4, N2-N2, CH4-CH4, H2-CH4
 * rtb_load_para_cia reads the same from the unformatted sequential file
 * fpread_all.f:45-97 reads (records: temps, fp, kh2h2, kh2he, kcia5). */
/* Load the exponential-integral table of e3interp (radtran/radtran/
 * e3interp.f:1-79; the e3tab.dat file it reads): n = 1001 transmissions
 * 0, 0.001, .., 1 and E3 at each (DOUBLE).  Needed by IMOD 18 paths
 * (hemispherically integrated emission, cirsradg_wave.f:1116-1225).
 * rtb_load_e3_table reads the text file (n, a header line, then n lines
 * tau tran e3). */
int rtb_set_e3_table(rtb_context* ctx, int n, const double* tran, const double* e3);
int rtb_load_e3_table(rtb_context* ctx, const char* path);

/* The stellar spectrum of /solardat/ (radtran/cirsrad/init_solar_wave.f:
 * 1-93; its presence is the reference's iread = 999): npt points wave[]
 * (the calculation's wavespace, monotonic) and rad[] (the star's total
 * power spectrum).  With it, iform = 1 divides the total planet flux of
 * IMOD 3 and 18 paths by get_solar_wave(v, -1) (cirsradg_wave.f:919-926,
 * 1142-1149) and iform = 4 multiplies IMOD 0 transmissions by
 * get_solar_wave(v, atm->dist) (:861-879); get_solar_wave.f:17-39 takes the
 * linear interpolation of interp.f, zero outside the table.  Without it both
 * factors are left out, as there.  rtb_load_stellar_spectrum reads the
 * text file (comment lines starting '#', the wavespace, which must equal
 * ispace, the stellar radius, then wave rad pairs). */
int rtb_set_stellar_spectrum(rtb_context* ctx, int npt, const float* wave, const float* rad);
int rtb_load_stellar_spectrum(rtb_context* ctx, const char* path, int ispace);

int rtb_set_para_cia(rtb_context* ctx, float dnu2, int ipara, const float* temps, const float* fp,
                     const float* kh2h2, const float* kh2he, const float* kcia5);
int rtb_load_para_cia(rtb_context* ctx, const char* path, float dnu2, int ipara);

/* The reference's table files, read on the host (no device work):
 * rtb_load_ktables reads ntab .kta files (read_klist.f / read_khead.f:33-110
 * header, then the records from IREC0 on) and loads them with
 * rtb_set_ktables; the tables must share the P, T and g grid (the /INTERPK/
 * block of get_kg.f:100-101); irregular tables (DELV <= 0) share DELV and
 * have their centres (VCEN records) within 1e-4 per cent of the first
 * table's (read_klist.f:160-176), which are loaded with
 * rtb_set_ktable_centres.  idgas/isogas
 * (may be NULL) receive each file's gas and isotope ids.
 * rtb_kta_header reads one header (no context needed).
 * rtb_load_cia reads a CIA .tab file (ciaread.f:77-98: sequential
 * unformatted, 25 DOUBLE temperatures then REAL kcia(9,25,1501)) and loads it
 * with rtb_set_cia. */
int rtb_kta_header(const char* path, int* np, int* nt, int* ng, int* npoint, float* vmin, float* delv,
                   int* idgas, int* isogas);
int rtb_load_ktables(rtb_context* ctx, int ntab, const char* const* paths, int* idgas, int* isogas);
int rtb_load_cia(rtb_context* ctx, const char* path, float dnu);

/* ---------------------------------------------------------------------- */
/* Forward model + Jacobian (cirsrtfg_wave replacement)                    */
/* ---------------------------------------------------------------------- */

/* The channels of the instrument convolution, cirsconv (radtran/cirsrad/
 * cirsconv.f:12-246), as cirsrtfg_wave hands them over (vconv, nconv and the
 * .fwh / .fil files it reads, cirsrtfg_wave.f:185-198, cirsconv.f:183-196). */
typedef struct rtb_conv {
    int nconv;
    const float* vconv;      /* (nconv) channel centres */
    /* FWHM > 0 only: the channel-dependent bin width of a .fwh file
     * (FWHMEXIST), VERINT-interpolated at each channel; nfwhm = 0 for none */
    int nfwhm;
    const float* vfwhm;      /* (nfwhm) */
    const float* xfwhm;      /* (nfwhm) */
    /* FWHM < 0 only: the filter functions of a .fil file; filter k is centred
     * at vcen[k] and has nsub[k] points (vfil, fil), filters concatenated */
    int nfil;
    const float* vcen;       /* (nfil) */
    const int* nsub;         /* (nfil) */
    const float* vfil;       /* (sum nsub) */
    const float* fil;        /* (sum nsub) */
} rtb_conv;

/* One call of cirsrtfg_wave after its set-up (subpathg + read_klist): the
 * layer/path arrays of /LAYCOM/ and /PATHCOM/, the gradient matrices of
 * /LGRAD/ and the state mapping xmap, by pointer, in Fortran layout.
 * Mirrors radtran/cirsradg/cirsrtfg_wave.f:1-3 (arguments :125-134) with the
 * implicit COMMON inputs made explicit. */
typedef struct rtb_atm {
    /* sizes */
    int nlayer, ngas, ncont, npath, npro, nv, nwave;
    /* leading dimensions of the Fortran arrays; 0 selects the reference
     * default (MAXLAY, MAXCON, MAXV, MAXGAS+2+MAXCON) */
    int ld_lay, ld_con, ld_v, ld_param;
    /* /LAYCOM/ (radtran/includes/laycom.f) */
    const float* press;    /* (nlayer) atm */
    const float* temp;     /* (nlayer) K */
    const float* delh;     /* (nlayer) km */
    const float* pp;       /* (ld_lay, ngas) atm */
    const float* amount;   /* (ld_lay, ngas) molecules cm-2 */
    const float* cont;     /* (ld_con, nlayer) particles cm-2 (ncont > 0) */
    const int*   idgas;    /* (ngas) */
    const int*   isogas;   /* (ngas) */
    /* gas -> k-table index loaded by rtb_set_ktables; -1 = no table (lun < 0);
     * RTB_KTAB_BY_ID = every loaded table of the gas's (idgas, isogas), in
     * load order, as read_klist assigns them per wavenumber */
    const int*   ktab;     /* (ngas) */
    /* /PATHCOM/ */
    const int*   nlayin;   /* (npath) */
    const int*   imod;     /* (npath) */
    const int*   layinc;   /* (ld_lay, npath), 1-based layer numbers */
    const float* scale;    /* (ld_lay, npath) */
    const float* emtemp;   /* (ld_lay, npath) K */
    /* /LGRAD/ (radtran/includes/laygrad.f:14-17) */
    const float* dte;      /* (ld_lay, npro) */
    const float* dam;      /* (ld_lay, npro) */
    const float* dco;      /* (ld_lay, npro), may be NULL when ncont == 0 */
    const float* dfp;      /* (ld_lay, npro), the para-H2 fraction's d(layer)/d(level), flagh2p = 1 only */
    /* state-vector mapping (cirsrtfg_wave.f argument) */
    const float* xmap;     /* (ld_v, ld_param, npro) */
    /* spectral grid and per-wavenumber dust cross sections */
    const float* vwave;    /* (nwave) calculation wavenumbers (cm-1) */
    const float* xsec_ext; /* (ncont, nwave) extinction x-sections at vwave, may be NULL if ncont == 0 */
    /* flags and scalars */
    int   inormal, iray, itype, ispace, flagh2p, ilbl, inlte, iform;
    float tsurf, fwhm;
    int   nem;
    const float* vem;        /* (nem) */
    const float* emissivity; /* (nem) */
    /* instrument channels; NULL means FWHM = 0 with nconv = nwave (the
     * outputs are on the calculation grid) */
    const rtb_conv* conv;
    /* flagh2p = 1 (para-H2 CIA through the table of rtb_set_para_cia): the
     * para-H2 fraction of every layer (HFP, /LAYCOM/); its gradient
     * parameter is the last, ngas + 1 + ncont, mapped to levels by dfp */
    const float* hfp;      /* (nlayer) */
    /* iform = 3 (total spectral flux of the planet, x 1e-18): the planet's
     * radius RADIUS1 and the height added above it, radextra, in km
     * (cirsradg_wave.f:913-929, 1136-1152) */
    float radius1, radextra;
    /* inlte = 1 (/nlte_flags/ of the .nlte file, cirsrtfg_wave.f:200-214):
     * collisional rate k1 (1e-20 .. 1e-3, else RTB_ERR_ARG) and the
     * Einstein A of calc_nlte_t.f; unused for inlte = 0 and 2 */
    float nlte_k1, nlte_A;
    /* distance from the star in AU (cirsrtfg_wave.f argument DIST): iform = 4
     * scales the star's spectrum by 1 / (4 pi (dist AU)^2) when dist > 0 */
    float dist;
    /* The gas-continuum switches of /GASCONDEF/ (radtran/includes/gascom.f,
     * read from the .fla file by READFLAGS) that NGASCON tests per layer and
     * gas (radtran/radtran/ngascon.f:132-318, called from cirsradg_wave.f:
     * 590-611): IH2O (H2O id 1, any isotope), ICH4 (CH4 id 6), INH3 (NH3
     * id 11), IO3 (O3 id 3) -- the last three for isotope 0 or 1 -- and the
     * iuvscat bitmask of UV cross sections (bit 1 NH3 11, 2 PH3 28, 4 C2H2
     * 26, 8 C2H6 27, 16 C4H2 30, 32 CH4 6, 64 CO 5, 128 GeH4 33, 256 H2O 1,
     * 512 C3H8 34).  A switch whose gas is absent contributes nothing, as in
     * the reference.  A switch whose gas is present would add a continuum
     * from data tables this library does not hold, so the call is refused
     * with RTB_ERR_UNSUPPORTED naming the switch and the gas; zero (the
     * reference's default) for all five is the computed path. */
    int ih2o, ich4, inh3, io3, iuvscat;
} rtb_atm;

/* Outputs, convolved by cirsconv with atm->fwhm onto the channels of
 * atm->conv (nconv = nwave when conv is NULL) and packed as cirsrtfg_wave
 * packs them (cirsrtfg_wave.f:448-516):
 *   calcout[nconv*ipath + iconv]
 *   gradients[nconv*nv*ipath + nconv*iv + iconv]
 *   gradtsurf[nconv*ipath + iconv]            (may be NULL)                */
int rtb_cirsrtfg_wave(rtb_context* ctx, const rtb_atm* atm,
                      float* calcout, float* gradients, float* gradtsurf);

/* Batched form: `nspec` independent spectra (uneven nlayer, ngas, nwave,
 * emission angle) in one persistent launch replayed through a CUDA graph.
 * Output pointers are arrays of per-spectrum host pointers. */
int rtb_cirsrtfg_wave_batch(rtb_context* ctx, int nspec, const rtb_atm* atms,
                            float* const* calcout, float* const* gradients,
                            float* const* gradtsurf);

/* Instrument convolution, cirsconv (radtran/cirsrad/cirsconv.f:12-246), of
 * nser series y[nser][nwave] on the calculation grid vwave to the channels
 * of conv, yout[nser][conv->nconv]:
 *   FWHM > 0  a natural cubic spline of each series averaged over a square
 *             bin of width fwhm (or the .fwh width at the channel) by a
 *             20-point trapezoid, divided by fwhm;
 *   FWHM = 0  a copy of the first nconv points (nconv <= nwave);
 *   FWHM < 0  the mean of the series weighted by the channel's filter
 *             function (the last filter centred within 1e-5 of the channel;
 *             a channel without one is refused);
 *   nwave = 1 and FWHM != 0: 1 (cirsconv.f:45-54; nconv must be 1).
 * rtb_cirsrtfg_wave applies the same convolution to its outputs. */
int rtb_cirsconv_ex(rtb_context* ctx, float fwhm, int nwave, const float* vwave, int nser, const float* y,
                    const rtb_conv* conv, float* yout);
/* The same with channel centres only (FWHM >= 0; FWHM = 0 needs nconv ==
 * nwave). */
int rtb_cirsconv(rtb_context* ctx, int nwave, const float* vwave, int nser, const float* y, float fwhm,
                 int nconv, const float* vconv, float* yout);

/* The text files of the convolution, read on the host (no context needed):
 * rtb_read_fwh reads a .fwh file (cirsrtfg_wave.f:191-196: NFWHM, then NFWHM
 * lines VFWHM XFWHM); rtb_read_fil reads a .fil file (cirsconv.f:185-196:
 * NCONV1, then per filter VCENTRAL, NSUB and NSUB lines VFIL FIL).  Called
 * with NULL arrays they return the counts only (*n, or *nfil and *npts =
 * sum of nsub); otherwise cap is the capacity of the arrays (points) and a
 * larger file is refused with RTB_ERR_LIMIT. */
int rtb_read_fwh(const char* path, int* n, float* v, float* x, int cap);
int rtb_read_fil(const char* path, int* nfil, int* npts, float* vcen, int* nsub, float* vfil, float* fil,
                 int cap_fil, int cap_pts);

/* Per-wavenumber compatibility form of cirsradg_wave (radtran/cirsradg/
 * cirsradg_wave.f:1-5, outputs :1240-1267) for A/B checks against the
 * reference one wavenumber at a time: the layer and path arrays as for
 * rtb_cirsrtfg_wave with atm->nwave == 1 (xmap, dte, dam, dco, npro and nv are
 * ignored), the active parameters isw[nsw] (0-based parameter ids: gases
 * 0..ngas-1, temperature ngas, dust ngas+1..; increasing, nsw <= 8; at
 * most 4 paths, RTB_ERR_UNSUPPORTED beyond) and:
 *   output[npath]           radiance of every path
 *   gtsurf[npath]           d output / d tsurf (may be NULL)
 *   doutputdq(ld_pat, ld_lay, ld_param)  d output(ipath) / d q(layer j of the
 *                           path, parameter k), zero outside isw, as the
 *                           reference's doutputdq(maxpat, maxlay, ...).
 * One wavenumber per call keeps the GPU mostly idle; rtb_cirsrtfg_wave is
 * the form to use for whole spectra. */
int rtb_cirsradg_wave(rtb_context* ctx, const rtb_atm* atm, int nsw, const int* isw, float* output,
                      float* gtsurf, float* doutputdq, int ld_pat, int ld_lay, int ld_param);

/* The same call split in three, for callers that keep a batch resident on
 * the device and replay it (a retrieval re-running its forward model, a
 * benchmark timing the kernel alone):
 *   rtb_fwd_prepare  validate, pack and upload the batch (synchronous);
 *   rtb_fwd_launch   run the forward kernel on the resident batch,
 *                    asynchronously on the context's stream;
 *   rtb_fwd_fetch    wait, then copy the outputs to the caller's buffers.
 * rtb_set_stream makes the context issue its work on a caller-owned CUDA
 * stream (a cudaStream_t passed as an opaque pointer; NULL restores the
 * context's own stream). */
int rtb_fwd_prepare(rtb_context* ctx, int nspec, const rtb_atm* atms);
int rtb_fwd_launch(rtb_context* ctx);
int rtb_fwd_fetch(rtb_context* ctx, float* const* calcout, float* const* gradients,
                  float* const* gradtsurf);
int rtb_set_stream(rtb_context* ctx, void* stream);

/* Diagnostics of the last forward call: (wavenumber, layer) cells, overlap
 * passes that sorted, passes with tied sort keys, passes that took the
 * reference heapsort (a tie that could move a g-bin boundary, a NaN key, or
 * every tie under rtb_set_strict_ties), passes whose g-walk crossed two
 * boundaries in one element (handled sequentially), and the device time of
 * the forward kernel. */
typedef struct rtb_fwd_stats {
    long long cells, sort_passes, tie_passes, exact_passes, irregular_passes;
    long long block_passes;           /* passes sorted by row-block ranks (no merge) */
    long long h2d_bytes, d2h_bytes;   /* host<->device bytes of the call */
    float ms_kernel;
    int grid;                         /* blocks of the last forward launch */
} rtb_fwd_stats;
int rtb_get_fwd_stats(const rtb_context* ctx, rtb_fwd_stats* out);

/* Debug capture for bit-exactness checks of the integer g-bin assignment.
 * With rtb_set_debug(ctx, 1) the next forward call records, for every
 * (wavenumber, layer, overlap pass igas = 1..ngas-1) of spectrum 0:
 *   perm  [iwave][ilayer][igas-1][ng*ng]  the sorted order of the combined
 *         elements (element i*ng + j: i over the accumulated distribution,
 *         j over the added gas, 0-based; noverlapg.f:117-125 loop order)
 *   split [iwave][ilayer][igas-1][ng]     the sorted position of the element
 *         at which g-bin b is closed (rankg.f:129-141), -1 if never closed.
 * Passes that do not sort (a zero distribution, noverlapg.f:88-108) hold -1.
 * n_perm / n_split are the element counts of the caller's buffers. */
int rtb_set_debug(rtb_context* ctx, int on);
int rtb_get_debug_bins(const rtb_context* ctx, int16_t* perm, size_t n_perm,
                       int16_t* split, size_t n_split);

/* Exact-heapsort policy for passes with tied sort keys: 0 (default) takes the
 * reference heapsort only where the order of tied keys can move a g-bin
 * boundary; 1 takes it for every pass that has a tie. */
int rtb_set_strict_ties(rtb_context* ctx, int on);

/* Schedule of the resident batch's launches.  A launch runs one block per
 * (spectrum, wavenumber) work item at a time on nsm x blocks_per_sm resident
 * blocks:
 *   schedule 0  static: block b takes items b, b + grid, ...
 *   schedule 1  dynamic: blocks pull the next item from a counter
 *   schedule 2  dynamic, items issued longest first (spectra ordered by a
 *               cost model: layers x overlap passes x gradient columns)
 * blocks_per_sm 0 = the occupancy maximum.  Results do not depend on the
 * schedule (each item is computed by one block, in the same order). */
int rtb_fwd_set_schedule(rtb_context* ctx, int schedule, int blocks_per_sm);

/* Tile shape of the resident batch's launches: warps per block, i.e. the
 * layers of one (spectrum, wavenumber) item worked on at once (one warp per
 * layer, one lane per g-ordinate): 2, 4 or 8; 0 = the default 8.  Tiles
 * other than 4 exist for the usual kernel instance (one temperature grid, no
 * para-H2 / IMOD 18 / iform / non-LTE / air-Rayleigh option); other batches
 * run 4.  Results do not depend on the tile. */
int rtb_fwd_set_tile(rtb_context* ctx, int warps);

/* Time the resident batch under every tile (2, 4, 8 warps per block) x
 * schedule x the three highest occupancies of the tile (two launches each,
 * the second timed), keep the fastest and report it.  The result is also
 * kept in the context under the batch's shape (its largest layer count in
 * buckets of 20 layers, and its largest gas count): a later rtb_fwd_prepare
 * of a batch of the same shape starts with it (tune on a representative
 * batch, run the large one).  rtb_fwd_set_schedule / rtb_fwd_set_tile after
 * the prepare override it; a batch of a shape not tuned in the context runs
 * the values last set with them (or the defaults). */
typedef struct rtb_fwd_tune {
    int schedule;
    int blocks_per_sm;
    float ms;          /* launch time of the chosen configuration */
    int candidates;    /* configurations timed */
    int warps;         /* warps per block of the chosen tile */
} rtb_fwd_tune;
int rtb_fwd_autotune(rtb_context* ctx, rtb_fwd_tune* out);

/* on = 1: rtb_fwd_launch replays a CUDA graph of one launch (status clear +
 * forward kernel), captured at the first launch after rtb_fwd_prepare or a
 * schedule change; on = 0: plain launches. */
int rtb_fwd_use_graph(rtb_context* ctx, int on);

/* ---------------------------------------------------------------------- */
/* Layering: profile -> layers and gradient matrices (subpathg set-up)     */
/* ---------------------------------------------------------------------- */

/* The atmospheric profile LAYERG integrates (the .prf arrays of /PATHCOM/
 * that subpathg reads: H, P, T, VMR, DUST, with RADIUS and MOLWT), by
 * pointer, in Fortran layout. */
typedef struct rtb_profile {
    int npro, nvmr, ndust;
    int ld_pro, ld_con;     /* leading dimensions of vmr and dust; 0 = npro, ndust */
    const float* h;         /* (npro) km, ascending */
    const float* p;         /* (npro) atm */
    const float* t;         /* (npro) K */
    const float* vmr;       /* (ld_pro, nvmr) volume mixing ratios */
    const float* dust;      /* (ld_con, npro) particles per gram of atmosphere; NULL if ndust == 0 */
    float molwt;            /* g/mol (AMFORM = 0) */
    float radius;           /* planet radius, km */
} rtb_profile;

/* The layering and path keywords of the .pat file (layerg.f:78-126 NLAY,
 * LAYTYP, LAYINT, LAYHT, LAYANG; atmg.f NADIR angle botlay ipzen, THERM,
 * BINBB).  laytyp 0 equal pressure, 1 equal log pressure, 2 equal height,
 * 3 equal path distance, 4 base pressures given (base, nlay values; the
 * pressure.lay file), 5 base heights given (height.lay); layint 0 layer-
 * centre values, 1 Curtis-Godson integration (101-point Simpson).  The path
 * is one nadir thermal-emission path (IMOD 3) through layers botlay..nlay at
 * `angle` degrees from the nadir (> 90 looks up from the bottom, atmg.f:
 * 142-147), with ipzen 0 (angle at the bottom layer) or 1 (angle defined at
 * 0 km, atmg.f:253-257). */
typedef struct rtb_layer_opts {
    int nlay, laytyp, layint;
    float layht, layang;
    const float* base;      /* laytyp 4 / 5: (nlay) base pressures (atm) / heights (km) */
    float angle;
    int botlay;             /* 1-based */
    int ipzen;
} rtb_layer_opts;

/* Outputs, in the layout of /LAYCOM/, /LGRAD/ and /PATHCOM/ (caller-owned
 * host arrays; NULL skips one).  Layer i is the i-th from the bottom. */
typedef struct rtb_layers {
    int ld_lay, ld_con;     /* leading dimensions of the 2-D outputs; 0 = nlay, ndust */
    float* baseh;           /* (nlay) km */
    float* delh;            /* (nlay) km */
    float* basep;           /* (nlay) atm */
    float* baset;           /* (nlay) K */
    float* press;           /* (nlay) atm, Curtis-Godson */
    float* temp;            /* (nlay) K */
    float* totam;           /* (nlay) molecules cm-2 (vertical path) */
    float* laysf;           /* (nlay) path / vertical length */
    float* amount;          /* (ld_lay, nvmr) */
    float* pp;              /* (ld_lay, nvmr) atm */
    float* cont;            /* (ld_con, nlay) particles cm-2 */
    float* dte;             /* (ld_lay, npro) d temp / d T(level) */
    float* dam;             /* (ld_lay, npro) d amount / d vmr(level) */
    float* dco;             /* (ld_lay, npro) d cont / d dust(level) */
    /* the path (atmg.f:290-373, 509-560) */
    int* npath;             /* 1 */
    int* nlayin;            /* (1) */
    int* imod;              /* (1) 3 */
    int* layinc;            /* (nlay) 1-based layers, farthest from the observer last */
    float* scale;           /* (nlay) */
    float* emtemp;          /* (nlay) K */
} rtb_layers;

/* LAYERG (radtran/path/layerg.f:146-458) and the nadir path of ATMG
 * (radtran/path/atmg.f:290-373) on the device, one warp per layer.  A layer
 * with a negative pressure, temperature, amount or dust column (the
 * reference's STOP at layerg.f:460-495) is refused with RTB_ERR_RANGE. */
int rtb_layerg(rtb_context* ctx, const rtb_profile* prof, const rtb_layer_opts* opts, rtb_layers* out);

/* ---------------------------------------------------------------------- */
/* Optimal-estimation Newton step (calc_gain_matrix + calcnextxn)          */
/* ---------------------------------------------------------------------- */

/* How the device forms K^T Se^-1 K:
 *   RTB_HESS_TC   tensor cores: Se^-1/2 K split into bf16 hi + lo parts,
 *                 three products per tile, FP32 accumulation; then `refine`
 *                 steps of iterative refinement in FP64 (default, refine 1);
 *   RTB_HESS_FP64 FP64 on the CUDA cores (the all-FP64 solve).
 * The Cholesky factorisation and the solves are FP64 in both. */
#define RTB_HESS_TC   0
#define RTB_HESS_FP64 1
int rtb_set_newton_mode(rtb_context* ctx, int hessian, int refine);

/* rtb_newton_step_batch -- the Newton step of nret independent retrievals
 * with diagonal Se (nemesis/calc_gain_matrix.f:123-163 for nx < ny, with
 * radtran/matrices/dinvertm.f jmod=2, then nemesis/calcnextxn.f:64-104):
 *     x_out = xa + D (y - yn) - AA (xa - xn)
 * computed as xa + C^-1 K^T Se^-1 (y - yn + K (xn - xa)), C = K^T Se^-1 K +
 * Sa^-1, without forming D or AA.  All arrays are host memory, retrieval r at
 * r * (its size):
 *   kk     [nret][nx][ny]  K^T: the `gradients` packing of rtb_cirsrtfg_wave
 *                          for one path, i.e. Fortran kk(ny, nx) with leading
 *                          dimension ny
 *   sei    [nret][ny]      diagonal of Se^-1 (the reference's dense sei(my,my)
 *                          is diagonal in every NEMESIS caller)
 *   sai    [nret][nx][nx]  Sa^-1
 *   xa, xn [nret][nx], y, yn [nret][ny]
 *   x_out  [nret][nx]      out
 *   nonpd  [nret]          out, may be NULL: 1 where a Cholesky pivot was <= 0
 *                          and replaced by 1 (dcholdc.f:69-84; the reference
 *                          continues the same way)
 *   resid  [nret]          out, may be NULL: ||rhs - C dx|| / ||rhs|| of the
 *                          final solve, C applied in FP64
 * 1 <= nx <= 128 on the device (NX = 124 at full size), nx < ny. */
int rtb_newton_step_batch(rtb_context* ctx, int nret, int nx, int ny, const float* kk, const double* sei,
                          const double* sai, const float* xa, const float* xn, const float* y,
                          const float* yn, float* x_out, int* nonpd, double* resid);

/* Device time of the last rtb_newton_step_batch kernel (Newton step of
 * `retrievals` retrievals, transfers excluded). */
typedef struct rtb_newton_stats {
    long long retrievals;
    float ms_kernel;
} rtb_newton_stats;
int rtb_get_newton_stats(const rtb_context* ctx, rtb_newton_stats* out);

/* calc_phiret (nemesis/calc_phiret.f:49-102) for nret retrievals, diagonal
 * Se: phi = (yn-y)^T Se^-1 (yn-y) + (xn-xa)^T Sa^-1 (xn-xa), chisq = the
 * first term, both REAL as in the reference.  Layouts as above. */
int rtb_calc_phiret_batch(rtb_context* ctx, int nret, int nx, int ny, const float* y, const float* yn,
                          const double* sei, const float* xn, const float* xa, const double* sai,
                          float* phi, float* chisq);

/* The reference's own interface for one retrieval, on the device in FP64:
 * calc_gain_matrix (nemesis/calc_gain_matrix.f:1-163, the nx < ny branch) with
 * a diagonal Se:
 *   kk   REAL kk(ldy, nx), column-major (Fortran kk_in): K(i, j) = dy_i / dx_j
 *   sxi  DOUBLE sxi(ldx, nx): Sa^-1
 *   sei  DOUBLE sei(ny): diagonal of Se^-1
 *   dd   DOUBLE dd(ldx, ny), out: gain matrix D = (K^T Se^-1 K + Sa^-1)^-1 K^T Se^-1
 *   aa   DOUBLE aa(ldx, nx), out: averaging kernels AA = D K
 *   nonpd  out, may be NULL: a Cholesky pivot was <= 0 (dcholdc.f:69-84)
 * and calcnextxn (nemesis/calcnextxn.f:1-109): x_out = x0 + D (y - yn) -
 * AA (x0 - xn) with D, AA as returned above.  Both run every product on the
 * device; rtb_newton_step_batch is the batched form that never forms D. */
int rtb_calc_gain_matrix(rtb_context* ctx, int nx, int ny, int ldx, int ldy, const float* kk,
                         const double* sxi, const double* sei, double* dd, double* aa, int* nonpd);
int rtb_calcnextxn(rtb_context* ctx, int nx, int ny, int ldx, const float* x0, const float* xn,
                   const float* y, const float* yn, const double* dd, const double* aa, float* x_out);
/* calc_serr (nemesis/calc_serr.f) after the last iteration, diagonal Se:
 * sm = D Se D^T (measurement error), sn = (AA - I) Sa (AA - I)^T (smoothing
 * error), st = sn + sm; sx REAL(ldx, nx), se REAL(ny) (the diagonal of
 * se_in), dd and aa as from rtb_calc_gain_matrix; outputs REAL(ldx, nx). */
int rtb_calc_serr(rtb_context* ctx, int nx, int ny, int ldx, const float* sx, const float* se,
                  const double* dd, const double* aa, float* st, float* sn, float* sm);

/* dinvertm (radtran/matrices/dinvertm.f jmod=2): inverse of nret symmetric
 * positive-definite n x n matrices (row-major, a[r*n*n]) by an FP64 Cholesky
 * factorisation on the device; n <= 128.  nonpd as above. */
int rtb_spd_inverse_batch(rtb_context* ctx, int nret, int n, const double* a, double* ainv, int* nonpd);

/* ---------------------------------------------------------------------- */
/* Retrieval loop (coreret Levenberg-Marquardt iteration)                  */
/* ---------------------------------------------------------------------- */

/* One retrieval of the layer-state model: the state vector is
 *   x[l]          temperature of layer l, l < nlayer (model 0, one level
 *                 per layer: DTE = identity, npro = nlayer)
 *   x[nlayer + a] a scale factor of gas scale_gas[a]: model 3 (default,
 *                 nemesis/subprofretg.f:735-750) the natural log of the
 *                 factor, amount, pp and the gas's xmap rows those of `atm`
 *                 times exp(x); model 2 (subprofretg.f:725-733) the factor
 *                 itself, amount and pp times x, xmap rows unchanged
 *   x[nlayer + nscale + p*nlayer + l]  natural log of the vmr of gas
 *                 prof_gas[p] in layer l (model 0 for a gas,
 *                 subprofretg.f:638-651): vmr = exp(x), the layer's amount
 *                 and pp those of `atm` times vmr / vmr_atm (vmr_atm = pp /
 *                 press), xmap row (l, gas, level l) = vmr
 * so nx = nlayer + nscale + nprof * nlayer.  `atm` is the atmosphere at scale factor 1 (its
 * temp is replaced by x, emtemp follows temp through layinc of every path);
 * each of its paths has at most nlayer positions, and its xmap must hold the
 * matching derivatives (T rows 1, gas rows the gas's vmr per level).  Host
 * pointers; read during the call only. */
typedef struct rtb_retrieval_spec {
    const rtb_atm* atm;
    int nscale;
    const int* scale_gas;     /* [nscale] 0-based gas index into atm */
    const float* y;           /* [ny] measurement: ny = npath x nwave, one spectrum per
                                 path, path after path (the level-state model has one
                                 path); with channels (atm->conv, any FWHM) nconv in
                                 place of nwave: every spectrum and Jacobian row is
                                 convolved onto them */
    const double* sei;        /* [ny] diagonal of Se^-1 */
    const double* sa;         /* [nx][nx] a priori covariance */
    const float* xa;          /* [nx] a priori state */
    const float* x0;          /* [nx] first guess; NULL = xa */
    const int* scale_model;   /* [nscale] 3 or 2; NULL = all 3 */
    int nprof;                /* gases retrieved as layer profiles */
    const int* prof_gas;      /* [nprof] 0-based gas index (not also in scale_gas) */
    /* The level-state model (NULL: the layer-state model above).  The state
     * is that of the profile's npro levels: x[lev] the temperature of level
     * lev, x[npro + a] the scale factor of gas scale_gas[a] (models 3 / 2 on
     * every level's vmr, subprofretg.f:725-750), x[npro + nscale + p*npro +
     * lev] the log vmr of gas prof_gas[p] at level lev (model 0); nx = npro +
     * nscale + nprof*npro.  Every state the loop evaluates rewrites the
     * profile and re-layers it on the device (rtb_layerg with lopts: layers,
     * DTE/DAM and the nadir path), the step gsetrad + subpathg take through
     * the .prf file each iteration; the Jacobian reaches the levels through
     * DTE/DAM and xmap (map2pro, map2xvec).  `atm` then supplies the gases
     * (ngas = prof->nvmr, idgas, isogas, ktab), the spectral grid and the
     * flags; its layer, path and gradient arrays and xmap are not read (may
     * be NULL); prof->ndust must be 0. */
    const rtb_profile* prof;
    const rtb_layer_opts* lopts;
    /* layer-state model: dust types whose column profile is scaled (model 3
     * on an aerosol, subprofretg.f:735-750): x[nlayer + nscale + nprof*nlayer
     * + d] is the log scale of dust type dust_type[d] (0-based, < ncont):
     * cont = cont_atm * exp(x); atm->xmap holds the matching rows (row d,
     * parameter ngas+1+type, level l: the type's column in layer l at scale
     * 1) and atm->dco maps layers to levels; nx grows by ndust */
    int ndust;
    const int* dust_type;
} rtb_retrieval_spec;

typedef struct rtb_retrieval_opts {
    int kiter;                /* Newton iterations (coreret.f:592 loop bound) */
    float phlimit;            /* convergence limit on the % change of phi (coreret.f:1003) */
    float dchisq_stop;        /* > 0: also stop when |chisq change| < this after an accepted step
                                 (a rule the reference does not have); <= 0: off */
    int max_batch;            /* retrievals resident at once (0 = all) */
} rtb_retrieval_opts;

typedef struct rtb_retrieval_result {
    float* x;                 /* [nx] out: final state (caller buffer) */
    float* yn;                /* [ny] out: spectrum at x (caller buffer, may be NULL) */
    float phi, chisq;         /* cost and chi^2 at x (calc_phiret) */
    float alambda;            /* final Marquardt brake */
    int iterations;           /* iterations taken */
    int forwards;             /* forward-model evaluations, the first included */
    int converged;            /* 0 kiter reached, 1 phlimit rule, 2 coreret.f:1022-1062
                                 alternate rule, 3 dchisq_stop */
    int nonpd;                /* a Cholesky pivot was replaced in some step */
    double ms;                /* wall time from submission (start of the call) to completion */
} rtb_retrieval_result;

/* Run nret retrievals to completion.  All retrievals iterate together: each
 * round runs one Newton step on the device for every retrieval whose K
 * changed, then one batched forward+Jacobian launch for every trial state,
 * then the cost on the device, and the coreret decision per retrieval
 * (accept: alambda *= 0.3; reject: *= 10, cap 1e10; trial states with a NaN,
 * a log variable beyond +-85, a negative model-2 scale or T < 1 are rejected
 * before the forward model, coreret.f:642-790).
 * K, spectra, Se^-1, Sa^-1 and the states stay in device memory between
 * rounds. */
int rtb_retrieve_batch(rtb_context* ctx, int nret, const rtb_retrieval_spec* specs,
                       const rtb_retrieval_opts* opts, rtb_retrieval_result* results);

/* ---------------------------------------------------------------------- */
/* Retrieval server (continuous batching)                                  */
/* ---------------------------------------------------------------------- */

/* A request loop over the same engine: requests are submitted at any time,
 * admitted first come first served whenever their device state fits in the
 * arena of hbm_budget_bytes (K of the current and the trial state, the
 * measurement and the two spectra, Se^-1, Sa, Sa^-1), and join the next
 * round; each round runs one batched Newton step, one batched
 * forward+Jacobian launch over every request in flight, whatever its size,
 * and the costs.  A request's result does not depend on what else is in
 * flight.  One host thread drives a server (submit, step, poll). */
typedef struct rtb_server rtb_server;
int  rtb_server_create(rtb_context* ctx, size_t hbm_budget_bytes, const rtb_retrieval_opts* opts,
                       rtb_server** out);
void rtb_server_destroy(rtb_server* srv);
/* copies the inputs (they may be freed on return); RTB_ERR_BUDGET if the
 * request could never fit the budget */
int  rtb_server_submit(rtb_server* srv, const rtb_retrieval_spec* spec, long long* id);
/* one round; reports the requests in flight and waiting */
int  rtb_server_step(rtb_server* srv, int* active, int* queued);
/* *done = 1 and the result (x, yn into the caller's buffers; ms = latency
 * from submission to completion) once request id has finished; each result
 * is returned once */
int  rtb_server_poll(rtb_server* srv, long long id, int* done, rtb_retrieval_result* result);

/* rtb_fwd_launch_static -- rtb_fwd_launch without the context's scratch.
 * No counterpart in the reference (the reference has no device memory).
 *
 * Some callers must not allocate device memory at the moment they run the
 * forward model: an application that reserves its whole device-memory budget
 * at start-up and hands the library nothing more, or a retrieval or serving
 * loop that keeps cudaMalloc/cudaFree out of its steady state because those
 * calls can synchronise the device and stall every other stream on it.  This
 * entry point runs the forward kernel on the batch resident from
 * rtb_fwd_prepare and allocates nothing: the kernel's per-block scratch (the
 * optical depths and their derivatives for every layer of the wavenumber a
 * block is working on) comes from one array compiled into the library,
 * RTB_STATIC_SCRATCH_BYTES per device, instead of the context's scratch.
 * Outputs, status and statistics are read with rtb_fwd_fetch as usual.
 *
 * Only the launch is allocation-free: rtb_fwd_prepare, which runs at set-up,
 * still sizes and allocates the context's buffers (the packed batch, the
 * outputs and the ordinary per-block scratch), as for rtb_fwd_launch.
 * First call: the first call on each device looks up the array's device
 * address (cudaGetSymbolAddress, with that device current) and keeps it for
 * the process; make that first call before any stream capture is started.
 * The address is not looked up again: after cudaDeviceReset (or with another
 * CUDA context made current on the device) it is stale, so a process that
 * resets a device must not call this entry point on it again.
 * Limit: a batch whose per-block slot (layers x NG x (1 + gradient columns)
 * floats, plus the parked k-distributions of wavenumbers between two table
 * points) does not fit in RTB_STATIC_SCRATCH_BYTES is refused with
 * RTB_ERR_LIMIT; a batch whose slots fit fewer blocks than rtb_fwd_launch
 * would use runs on that many blocks (rtb_fwd_stats.grid).  Nothing in the array needs to start at
 * zero; the status and counter words that do are cleared on the stream by
 * every call.
 * Races: the array is one per device, shared by every context of the process
 * on that device.  Two calls whose kernels can overlap in time (different
 * streams, contexts or host threads on the same device) overwrite each
 * other's scratch; order them on one stream or with events. */
#define RTB_STATIC_SCRATCH_BYTES (32u << 20)
int rtb_fwd_launch_static(rtb_context* ctx);

#ifdef __cplusplus
}
#endif
#endif /* RADTRAN_B200_H */
