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
 *                   block of get_kg.f:100-101 does); nt > 0 only
 *   lnp[np]         log of the table pressures in atm (read_khead.f:81-84)
 *   tk[nt]          table temperatures, K
 *   delg[ng]        g-ordinate weights (DEL_G)
 *   vmin[ntab], delv[ntab], nbin[ntab]   wavenumber grid of each table
 *                   (delv > 0: regular grid as in get_kg.f:193-208)
 *   data            concatenation over tables of REAL k(ng, nt, np, nbin) in
 *                   record order: record = ((ibin*np + ip)*nt + it)*ng + ig,
 *                   i.e. exactly the .kta record order after IREC0, values
 *                   multiplied by 1e20 as stored in the files.
 * Tables stay resident until the next call or rtb_destroy. */
int rtb_set_ktables(rtb_context* ctx, int ntab, int np, int nt, int ng,
                    const float* lnp, const float* tk, const float* delg,
                    const float* vmin, const float* delv, const int* nbin,
                    const float* data);

/* Load a CIA table: replaces the one-time read of ciaread
 * (radtran/radtran/ciaread.f:63-105) into /CIATABLE/.
 *   dnu          wavenumber step of the table grid vvk1(i) = (i-1)*dnu
 *   temps[25]    DOUBLE temperatures as in the file's first record
 *   kcia         REAL kcia(9, 25, 1501), Fortran order (pair fastest). */
int rtb_set_cia(rtb_context* ctx, float dnu, const double* temps, const float* kcia);

/* ---------------------------------------------------------------------- */
/* Forward model + Jacobian (cirsrtfg_wave replacement)                    */
/* ---------------------------------------------------------------------- */

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
    /* gas -> k-table index loaded by rtb_set_ktables; -1 = no table (lun < 0) */
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
    const float* dfp;      /* (ld_lay, npro), unused (flagh2p must be 0) */
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
} rtb_atm;

/* Outputs, packed as cirsrtfg_wave packs them (cirsrtfg_wave.f:425-446,
 * FWHM = 0 so cirsconv is the identity and nconv = nwave):
 *   calcout[nwave*ipath + iwave]
 *   gradients[nwave*nv*ipath + nwave*iv + iwave]
 *   gradtsurf[nwave*ipath + iwave]            (may be NULL)                */
int rtb_cirsrtfg_wave(rtb_context* ctx, const rtb_atm* atm,
                      float* calcout, float* gradients, float* gradtsurf);

/* Batched form: `nspec` independent spectra (uneven nlayer, ngas, nwave,
 * emission angle) in one persistent launch replayed through a CUDA graph.
 * Output pointers are arrays of per-spectrum host pointers. */
int rtb_cirsrtfg_wave_batch(rtb_context* ctx, int nspec, const rtb_atm* atms,
                            float* const* calcout, float* const* gradients,
                            float* const* gradtsurf);

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
 * First call: the first call on each device looks up the array's device
 * address (cudaGetSymbolAddress, with that device current) and keeps it for
 * the process; make that first call before any stream capture is started.
 * Limit: a batch whose per-block slot (layers x NG x (1 + gradient columns)
 * floats) does not fit in RTB_STATIC_SCRATCH_BYTES is refused with
 * RTB_ERR_LIMIT; a batch whose slots fit fewer blocks than rtb_fwd_launch
 * would use runs on that many blocks.  Nothing in the array needs to start at
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
