// rtb_common.h -- data layout shared by the host orchestration (host.cu)
// and the forward kernel (fwd_kernel.cu).
//
// A launch processes a *batch* of spectra.  Every per-spectrum input is
// packed by the host into flat device arrays; a SpecDev descriptor holds the
// offsets.  Work items are (spectrum, wavenumber) pairs: one CTA per item.
#pragma once
#include <stdint.h>

namespace rtb {

constexpr int kMaxNg = 32;        // one lane per g-ordinate
constexpr int kMaxCols = 8;       // tracked gradient columns in the overlap (active gases + T)
constexpr int kMaxSw = 8;         // active Jacobian columns (isw) per spectrum
constexpr int kMaxGasDev = 30;    // MAXGAS
constexpr int kMaxPathDev = 4;    // paths of one spectrum per device work item (more: path groups)
constexpr int kWarps = 4;         // warps per CTA of the forward kernel (every instance has this tile)
constexpr int kTileDefault = 8;   // the tile a batch runs unless tuned or set (where its instance has it)
constexpr int kThreads = kWarps * 32;

// status bits accumulated by the kernel (OR-ed into a device word)
constexpr unsigned kStGord = 1u;       // g-walk ran past NG with elements left
constexpr unsigned kStNanKey = 2u;     // NaN sort key met (handled by the exact path)
constexpr unsigned kStRange = 4u;      // index outside a table

// per-layer constants prepared on the host (get_kg.f:117-141, ciaread.f:108-198,
// nciacon.f:84-177), identical arithmetic to the oracle
struct LayerDev {
    int ioff[4];          // offsets of the 4 (P,T) corners inside a (np,nt,ng) slice
    float u, v, dudt;     // get_kg interpolation weights
    float utotl;          // sum of amounts * 1e-20
    int cia_ct;           // CIA temperature index (0-based), -1 = no CIA
    float cia_u, cia_dudt;
    float cia_tau;        // height * amagat^2 of nciacon
    float q[5];           // qh2, qhe, qn2, qch4, qco2
    int iabs[5];          // 0-based gas index or -1
    float u2, dudt2;      // NT < 0: the temperature weight at pressure cp + 1 (get_kg.f:157-165)
};

// per-wavenumber constants
struct WaveDev {
    float vwave;          // calculation wavenumber
    int cia_cv;           // CIA wavenumber index (0-based), -1 = outside the table -> zero
    float cia_t;          // CIA wavenumber weight
    float xray;           // Rayleigh x-section * 1e20 (0 if off)
    float radground_s;    // esurf*B(tsurf) when tsurf > 0
    float gradground_s;   // esurf*dB/dT(tsurf)
};

// para-H2 CIA (flagh2p = 1, nparacon_all.f / fpread_all.f): per layer the
// table temperature bracket and the para-fraction bracket, per wavenumber the
// table wavenumber bracket
struct ParaLayDev {
    int ct;               // 0-based temperature index of fpread_all's PINDEX
    float u, dudt;
    int j0;               // 0-based lower para-fraction entry used
    float f;              // weight of the entry above it
    int neg;              // fpara < 0: entry j0 = KPARA alone, no para derivative
};

struct ParaWaveDev {
    int cv;               // 0-based wavenumber index
    float t;
};

// per-spectrum descriptor
struct SpecDev {
    int nlayer, ngas, npath, nwave, nv, ncont, nsw, nlmax;
    int ncol;             // tracked overlap columns
    int tsurf_pos;        // tsurf > 0
    float xfac3, xfac18;  // iform factor of the IMOD 3 and IMOD 18 paths (1 unless iform = 3)
    int inlte;            // non-LTE emission temperatures (calc_nlte_t.f): 0, 1 or 2
    float nlte_k1, nlte_A;
    int64_t lp_off;       // lay_press index of layer 0 (inlte != 0 or iray = 3)
    int64_t lt_off;       // lay_temp index of layer 0 (iray = 3)
    int wmode;            // stellar factor per wavenumber: 0 none, 1 divides (iform 1), 2 multiplies IMOD 0 (iform 4)
    int64_t wf_off;       // wave_fac index of wavenumber 0 (wmode != 0)
    int nonlimb_mask;     // bit p: path p adds the surface term (cirsradg_wave.f:985-1000)
    int ispace;
    int inormal;
    int iray;             // IRAY (1 Jovian, 2 Venus, 3 air) when ITYPE != 0, else 0
    int has_cia;
    int64_t lay_off;      // LayerDev index of layer 0
    int64_t lg_off;       // (layer, gas) arrays: index of (0,0); [nlayer][ngas]
    int64_t wave_off;     // WaveDev index of wavenumber 0
    int64_t wg_off;       // (wave, gas) arrays: [nwave][ngas] table slice offsets
    int64_t wc_off;       // (wave, cont) dust x-sections [nwave][ncont]
    int64_t lc_off;       // (layer, cont) dust amounts [nlayer][ncont]
    int64_t path_off;     // path-position arrays [npath][nlmax]
    int64_t map_off;      // map CSC: colptr index of (path 0, iv 0); [npath][nv+1]
    int64_t out_off;      // calcout/gradtsurf index of (path 0, wave 0)
    int64_t jac_off;      // gradients index of (path 0, iv 0, wave 0)
    int nlayin[kMaxPathDev];  // the spectrum's paths in this group
    int imod[kMaxPathDev];
    int isw[kMaxSw];      // active parameters (0-based param ids)
    int col_of_param[kMaxSw]; // tracked overlap column of isw[s] (-1: continuum only)
    int col_gas[kMaxCols];    // gas index of tracked column c (ngas = temperature)
    int sw_T;             // s index of the temperature column, -1 if inactive
    int para;             // flagh2p = 1: the para-H2 CIA replaces the CIA table
    int sw_para;          // s index of the para-H2 fraction column, -1 if inactive
    int64_t para_off;     // ParaLayDev index of layer 0 / ParaWaveDev index of wavenumber 0
    int64_t paraw_off;
};

struct BatchDev {
    int nspec;
    int64_t nitems;              // sum of nwave
    const int64_t* item_start;   // [nspec+1] prefix sum of nwave
    const SpecDev* spec;
    const LayerDev* lay;
    const float* amo;            // [.. nlayer][ngas] amount*1e-20
    const WaveDev* wave;
    const int64_t* wg_slice;     // [.. nwave][ngas] element offset of the table slice, -1 = zero
    const float* wg_w2;          // [.. nwave][ngas] non-coincident weight of slice+1 (< 0: coincident); may be null
    const float* wg_w1;          // [.. nwave][ngas] weight of slice (irregular grids); null: 1 - wg_w2
    const float* xsec;           // [.. nwave][ncont]
    const float* cont;           // [.. nlayer][ncont]
    const int* p_layinc;         // [.. npath][nlmax] 0-based layer
    const float* p_scale;
    const float* p_emtemp;
    const int* map_colptr;       // [.. npath][nv+1] into map_row/map_val (absolute)
    const int* map_row;          // s*nlmax + j
    const float* map_val;
    // tables
    const float* ktab_raw;       // k*1e20, record order
    const float* ktab_log;       // (float)log((double)k)
    int np, nt, ng;              // nt = |NT|
    int t2;                      // NT < 0: one temperature grid per pressure (TEMP2)
    const float* delg;           // [ng]
    const double* g_ord;         // [ng+1], g_ord[ng] forced >= 1 (rankg.f:65-67)
    const float* kcia;           // (9,25,1501) Fortran order
    // E3 table of e3interp (IMOD 18): tabtran | tabe3 | egrad, 1001 each
    const double* e3tab;
    // para-H2 CIA (spectra with flagh2p = 1)
    int para;                    // any spectrum of the batch uses it
    int ext;                     // para, an IMOD 18 path or iform = 3 somewhere in the batch
    int ipara;                   // tabulated para fractions
    float para_deltaf;           // fp(2) - fp(1)
    const float* kh2h2;          // (ipara,25,1501) Fortran order
    const float* kh2he;
    const float* kcia5;          // (5,25,1501)
    const ParaLayDev* para_lay;
    const ParaWaveDev* para_wave;
    const float* lay_press;      // [.. nlayer] layer pressures (atm) of non-LTE / air-Rayleigh spectra
    const float* lay_temp;       // [.. nlayer] layer temperatures (K) of air-Rayleigh spectra
    const float* wave_fac;       // [.. nwave] get_solar_wave of iform 1 / 4 spectra
    // per-CTA scratch slots (tau, dtau/dq of every layer of the current item)
    float* cell_scratch;
    int64_t cell_slot;             // floats per slot
    int cell_Lmax;                 // layers per slot
    int64_t nc_off;                // floats from the slot start to the non-coincident k area
                                   // [layer][gas][kMaxNg][2] (k, dk/dT), when wg_w2 is set
    // outputs
    float* calcout;
    float* gradients;
    float* gradtsurf;
    // diagnostics
    unsigned* status;
    unsigned long long* counters;  // [0] sort passes [1] tie passes [2] risky/exact passes [3] irregular
    int strict_ties;               // 1: exact heapsort for every pass with tied keys
    int16_t* dbg_perm;             // debug capture for spectrum 0 (may be null)
    int16_t* dbg_split;
    // schedule (autotuned): issue order of the items, and the dynamic
    // work counter (zero at launch; nullptr = static grid-stride)
    const int* item_order;
    unsigned long long* work_next;
    // per-path-position derivatives dR/dq (cirsradg_wave's doutputdq) of every
    // item, [wave][npath][dq_stride] with dq_stride = nlmax x nsw; nullptr = off
    float* dq_out;
    int64_t dq_stride;
    int dq_npath;
};

}  // namespace rtb
