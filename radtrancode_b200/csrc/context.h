// context.h -- internal: the device context behind the C ABI and the
// batch staging shared by the forward entry points (host.cu) and the
// retrieval engine (retrieval.cu).  Not installed; the public interface is
// include/radtran_b200.h.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <map>
#include <string>
#include <vector>

#include "../../include/radtran_b200.h"
#include "rtb_common.h"

namespace rtb {
int fwd_smem_bytes(int ng, int nsw, int ncol, int nlmax, int npath, int warps);
// warps per CTA a launch uses for a requested tile (tiles other than kWarps
// exist for the usual instance only), and the blocks per SM it can hold
int fwd_tile_warps(bool t2, bool ext, int warps);
int fwd_blocks_per_sm(int smem, bool t2, bool ext, int warps, int ng);
cudaError_t launch_fwd(const BatchDev& B, int nsw, int ncol, int nlmax, int npath, int grid, int warps,
                       cudaStream_t st);

// growable device buffer / pinned host buffer (grow-only, freed by release)
// growable device buffer
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t n) {
        if (n <= cap) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        size_t c = std::max(n, (size_t)4096);
        c = c + c / 4;
        cudaError_t e = cudaMalloc(&p, c);
        if (e == cudaSuccess) cap = c;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

struct HostPinned {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t n) {
        if (n <= cap) return cudaSuccess;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        size_t c = std::max(n, (size_t)4096);
        c = c + c / 4;
        cudaError_t e = cudaMallocHost(&p, c);
        if (e == cudaSuccess) cap = c;
        return e;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
    }
};

// host staging of one batch
struct Staging {
    std::vector<SpecDev> spec;
    std::vector<int64_t> item_start;
    std::vector<LayerDev> lay;
    std::vector<float> amo;
    std::vector<WaveDev> wave;
    std::vector<int64_t> wg_slice;
    std::vector<float> wg_w2;         // [.. nwave][ngas] upper-point weight, < 0 coincident
    std::vector<float> wg_w1;         // [.. nwave][ngas] lower-point weight of an irregular grid, < 0 none
    bool any_noncoinc = false;
    bool any_w1 = false;
    bool any_para = false;
    bool any_ext = false;        // an IMOD 18 path or iform = 3

    std::vector<float> xsec, cont;
    std::vector<int> p_layinc;
    std::vector<float> p_scale, p_emtemp;
    std::vector<int> map_colptr, map_row;
    std::vector<float> map_val;
    std::vector<ParaLayDev> para_lay;
    std::vector<ParaWaveDev> para_wave;
    std::vector<float> lpress;   // layer pressures (atm) of the spectra with non-LTE emission or air Rayleigh
    std::vector<float> ltemp;    // layer temperatures (K) of the spectra with air Rayleigh
    std::vector<int> nsub;       // device spectra (path groups) of each caller spectrum, in order
    std::vector<float> wfac;     // get_solar_wave at each wavenumber of iform 1 / 4 spectra
    int Lmax = 0, nsw_max = 1, ncol_max = 1, nlmax_max = 1, npath_max = 1, ngas_max = 1;
    int64_t n_out = 0, n_jac = 0;
};

// where a batch's outputs go: the context's own arena (nullptr) or caller
// device arrays, with per-spectrum element offsets
struct OutPlace {
    float* calcout;
    float* gradtsurf;
    float* gradients;
    const int64_t* out_off;   // [nspec] into calcout / gradtsurf
    const int64_t* jac_off;   // [nspec] into gradients
};

int fail(rtb_context* c, int code, const char* fmt, ...);
int pack_spectrum(rtb_context* c, const rtb_atm& a, Staging& st);
int prepare_ex(rtb_context* c, int nspec, const rtb_atm* atms, const OutPlace* place);
int launch(rtb_context* c);
int apply_schedule(rtb_context* c);
void drop_graph(rtb_context* c);
cudaStream_t stream_of(rtb_context* c);

// one spectrum's instrument convolution (the cirsconv arguments), copied
// when the batch is prepared
struct ConvSpec {
    float fwhm = 0.0f;
    std::vector<float> vwave, vconv;          // empty vconv: no convolution (FWHM = 0, nconv = nwave)
    std::vector<float> vfwhm, xfwhm;          // FWHM > 0: channel-dependent width table
    std::vector<int> fil_of, fil_off;         // FWHM < 0: filter of each channel; point offsets per filter
    std::vector<float> vfil, fil;
};
// nser device series of nwave values at y, convolved to yout[nser][nconv]
struct ConvSeg {
    const float* y;
    int nser;
    float* yout;
};
int conv_check(rtb_context* c, float fwhm, int nwave, const float* vwave, const rtb_conv* cv, ConvSpec& out);
int conv_run(rtb_context* c, const ConvSpec& cs, int nseg, const ConvSeg* seg, cudaStream_t st);

}  // namespace rtb

// the context is the opaque handle of the C ABI (global namespace)
struct rtb_context {
    int device = 0;
    int nsm = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::string err;
    // k-tables
    int ntab = 0, np = 0, nt = 0, ng = 0;
    std::vector<float> lnp, tk, delg;
    std::vector<double> g_ord;
    std::vector<float> vmin, delv;
    std::vector<int> nbin;
    std::vector<int64_t> tab_off;            // element offset of each table
    std::vector<float> vcen;                 // irregular grids: the first table's centres VCEN(NPOINT)
    std::vector<int> tab_id, tab_iso;        // the tables' gas and isotope ids (RTB_KTAB_BY_ID), empty: unknown
    std::vector<std::vector<uint8_t>> nonzero;  // [tab][bin]: any value > 0 (get_kg.f:228-250)
    rtb::DevBuf d_raw, d_log, d_delg, d_gord;
    // CIA
    int has_cia = 0;
    float dnu = 0.0f;
    // para-H2 CIA (fpread_all)
    int has_para = 0, ipara = 0;
    float dnu2 = 0.0f, para_deltaf = 0.0f;
    std::vector<float> para_tk, para_fp, para_vk;
    rtb::DevBuf d_kpara;                     // kh2h2 | kh2he | kcia5
    int has_e3 = 0;
    // /solardat/ (init_solar_wave): the stellar spectrum, used on the host only
    std::vector<float> solar_wave, solar_rad;
    rtb::DevBuf d_e3;                        // tabtran | tabe3 | egrad (e3interp)
    std::vector<float> cia_tk;               // sngl(temps)
    rtb::DevBuf d_kcia;
    // per-call arena
    rtb::DevBuf d_in, d_out, d_diag, d_cells;
    rtb::HostPinned h_in, h_out;
    // options and diagnostics
    int strict_ties = 0;
    int debug = 0;
    cudaStream_t user_stream = nullptr;   // caller-provided stream (NULL: own stream)
    // resident batch (rtb_fwd_prepare)
    int prepared = 0;
    int placed = 0;                       // outputs of the resident batch go to caller device arrays
    rtb::BatchDev B{};
    int Lmax = 0, nsw_max = 1, ncol_max = 1, nlmax_max = 1, npath_max = 1, grid = 1;
    std::vector<rtb::SpecDev> spec_host;
    std::vector<int> spec_npath, spec_nv, spec_nwave, spec_nlayer;
    int64_t n_out = 0, n_jac = 0;
    size_t in_bytes = 0, out_bytes = 0;
    long long cells = 0;
    rtb::DevBuf d_dbg_perm, d_dbg_split;
    rtb::DevBuf d_dq;                     // per-path-position derivatives (rtb_cirsradg_wave)
    // instrument convolution of the resident batch's outputs (cirsrtfg_wave.f:448-516)
    std::vector<rtb::ConvSpec> spec_conv;
    int any_conv = 0;
    rtb::DevBuf d_conv, d_convout;
    rtb::DevBuf d_layer;                  // rtb_layerg inputs, arguments and outputs
    std::vector<char> h_conv;
    size_t dbg_perm_n = 0, dbg_split_n = 0;
    rtb_fwd_stats stats{};
    int launched_grid = 0;                // blocks of the last forward launch
    // schedule of the resident batch (rtb_fwd_set_schedule / rtb_fwd_autotune)
    int sched = 0;                        // 0 static, 1 dynamic, 2 dynamic cost-ordered
    int occ = 0;                          // blocks per SM (0 = the occupancy maximum)
    int tile = rtb::kWarps;               // requested warps per CTA (rtb_fwd_set_tile / rtb_fwd_autotune)
    // the caller's own choices (rtb_fwd_set_tile / rtb_fwd_set_schedule), which a batch of an untuned shape uses
    int tile_user = rtb::kTileDefault, sched_user = 0, occ_user = 0;
    int tile_eff = rtb::kWarps;           // warps per CTA of the resident batch's launches
    int bpsm_w[9] = {};                   // blocks per SM of the batch at 2, 4, 8 warps per CTA (0: not resident)
    int bpsm_max = 1;                     // blocks per SM of the current tile
    // rtb_fwd_autotune results by batch shape (layer bucket of 20, gas count): tile, schedule, occupancy
    std::map<std::pair<int, int>, std::array<int, 3>> tuned;
    std::pair<int, int> shape{0, 0};      // shape of the resident batch
    std::vector<int64_t> item_start_host;
    std::vector<float> spec_cost;
    int order_ready = 0;
    rtb::DevBuf d_order;
    // CUDA graph of one launch of the resident batch (rtb_fwd_use_graph)
    int use_graph = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    // Newton step
    int newton_hess = 0;                  // RTB_HESS_TC / RTB_HESS_FP64
    int newton_refine = 1;
    rtb::DevBuf d_nt32, d_nt64, d_ntsmall, d_ntdesc;
    rtb_newton_stats newton_stats{};
};

#define CUDA_TRY(ctx, call)                                                                 \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return fail(ctx, RTB_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)
