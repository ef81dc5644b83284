// formats.cu -- the reference's table files, read on the host and handed to
// rtb_set_ktables / rtb_set_cia.
//
// .kta (radtran/cirsrad/read_khead.f:33-110, written by
// radtran/radtran/calc_fnktablec.f:304-367): a direct-access file of 4-byte
// records (RECL = ISYS() = 4 with gfortran).  Records, 1-based: 1 IREC0,
// 2 NPOINT, 3 VMIN, 4 DELV, 5 FWHM, 6 NP, 7 NT, 8 NG, 9 IDGAS, 10 ISOGAS,
// 11.. G_ORD(NG), DEL_G(NG), two spare records, PRESS(NP) in atm, TEMP(NT)
// (or TEMP2(NP,|NT|) when NT < 0), VCEN(NPOINT) when DELV <= 0; the k values
// (x 1e20) from record IREC0 on, bin by bin, (P, T, g) with g fastest
// (get_kg.f:137-140, 211, 293-296).
//
// CIA .tab (radtran/radtran/ciaread.f:77-98): a sequential unformatted file
// with two records, 25 DOUBLE temperatures and REAL kcia(9, 25, 1501), each
// framed by 4-byte length markers.
//
// .fwh and .fil (cirsrtfg_wave.f:185-198, cirsconv.f:183-196): text files
// read by list-directed READ(u,*), the channel widths and filter functions of
// the instrument convolution, handed to rtb_cirsconv_ex / rtb_conv.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "context.h"

namespace rtb {

namespace {

struct File {
    FILE* f = nullptr;
    explicit File(const char* p) : f(p ? std::fopen(p, "rb") : nullptr) {}
    ~File() {
        if (f) std::fclose(f);
    }
};

struct Kta {
    int irec0 = 0, npoint = 0, np = 0, nt = 0, ng = 0, idgas = 0, isogas = 0;
    float vmin = 0, delv = 0, fwhm = 0;
    std::vector<float> press, temp, delg, vcen;
};

// 1-based 4-byte record n of a direct-access file
bool rec4(FILE* f, long n, void* out) {
    if (std::fseek(f, (n - 1) * 4L, SEEK_SET) != 0) return false;
    return std::fread(out, 4, 1, f) == 1;
}

bool recs4(FILE* f, long n, size_t count, void* out) {
    if (std::fseek(f, (n - 1) * 4L, SEEK_SET) != 0) return false;
    return std::fread(out, 4, count, f) == count;
}

// read_khead.f:47-110; returns an RTB status, message in err
int read_kta_header(FILE* f, Kta& k, std::string& err) {
    bool ok = rec4(f, 1, &k.irec0) && rec4(f, 2, &k.npoint) && rec4(f, 3, &k.vmin) && rec4(f, 4, &k.delv) &&
              rec4(f, 5, &k.fwhm) && rec4(f, 6, &k.np) && rec4(f, 7, &k.nt) && rec4(f, 8, &k.ng) &&
              rec4(f, 9, &k.idgas) && rec4(f, 10, &k.isogas);
    if (!ok) {
        err = "short .kta header";
        return RTB_ERR_ARG;
    }
    if (k.np <= 0 || k.np > RTB_MAXK || k.ng <= 0 || k.ng > RTB_MAXG - 1 || k.npoint <= 0 || k.nt == 0 ||
        std::abs(k.nt) > RTB_MAXK) {
        err = "implausible .kta sizes (NP, NT, NG, NPOINT)";
        return RTB_ERR_LIMIT;
    }
    // TEMP(NT), or TEMP2(NP, |NT|) stored with the temperature index fastest
    // (read_khead.f:86-98); kept column-major (pressure fastest) as TEMP2 is
    const int ntk = k.nt > 0 ? k.nt : k.np * -k.nt;
    k.delg.resize(k.ng);
    k.press.resize(k.np);
    std::vector<float> rec(ntk);
    ok = recs4(f, 11 + k.ng, k.ng, k.delg.data()) && recs4(f, 11 + 2 * k.ng + 2, k.np, k.press.data()) &&
         recs4(f, 11 + 2 * k.ng + 2 + k.np, ntk, rec.data());
    if (!ok) {
        err = "short .kta header arrays";
        return RTB_ERR_ARG;
    }
    k.temp.resize(ntk);
    if (k.nt > 0) {
        k.temp = rec;
    } else {
        for (int i = 0; i < k.np; ++i)
            for (int j = 0; j < -k.nt; ++j) k.temp[i + (size_t)k.np * j] = rec[(size_t)i * -k.nt + j];
    }
    // the centres of an irregular grid (read_khead.f:100-103)
    const int nvc = k.delv > 0.0f ? 0 : k.npoint;
    if (nvc) {
        k.vcen.resize(nvc);
        if (!recs4(f, 11 + 2 * k.ng + 2 + k.np + ntk, nvc, k.vcen.data())) {
            err = "short .kta centre records";
            return RTB_ERR_ARG;
        }
    }
    if (k.irec0 < 11 + 2 * k.ng + 2 + k.np + ntk + nvc) {
        err = "IREC0 points into the .kta header";
        return RTB_ERR_ARG;
    }
    return RTB_OK;
}

// One list-directed READ(u,*) of n values (the Fortran rule the reference's
// text files rely on): it starts at the next record, takes values separated
// by blanks or commas across as many records as it needs, and drops the rest
// of its last record.
bool list_read(FILE* f, int n, std::vector<std::string>& out) {
    out.clear();
    char line[4096];
    while ((int)out.size() < n) {
        if (!std::fgets(line, sizeof line, f)) return false;
        std::string cur;
        for (const char* p = line;; ++p) {
            const char ch = *p;
            if (ch == ' ' || ch == '\t' || ch == ',' || ch == '\n' || ch == '\r' || ch == '\0') {
                if (!cur.empty() && (int)out.size() < n) out.push_back(cur);
                cur.clear();
                if (ch == '\0') break;
            } else {
                cur += ch;
            }
        }
    }
    return true;
}

bool to_int(const std::string& t, int& v) {
    char* e = nullptr;
    const long x = std::strtol(t.c_str(), &e, 10);
    if (e == t.c_str() || *e) return false;
    v = (int)x;
    return true;
}

bool to_real(std::string t, float& v) {
    for (char& ch : t)
        if (ch == 'd' || ch == 'D') ch = 'e';   // DOUBLE PRECISION exponent letter
    char* e = nullptr;
    v = std::strtof(t.c_str(), &e);
    return e != t.c_str() && !*e;
}

}  // namespace

}  // namespace rtb

using namespace rtb;

extern "C" {

int rtb_kta_header(const char* path, int* np, int* nt, int* ng, int* npoint, float* vmin, float* delv, int* idgas,
                   int* isogas) {
    File fl(path);
    if (!fl.f) return RTB_ERR_ARG;
    Kta k;
    std::string err;
    const int r = read_kta_header(fl.f, k, err);
    if (r) return r;
    if (np) *np = k.np;
    if (nt) *nt = k.nt;
    if (ng) *ng = k.ng;
    if (npoint) *npoint = k.npoint;
    if (vmin) *vmin = k.vmin;
    if (delv) *delv = k.delv;
    if (idgas) *idgas = k.idgas;
    if (isogas) *isogas = k.isogas;
    return RTB_OK;
}

int rtb_load_ktables(rtb_context* c, int ntab, const char* const* paths, int* idgas, int* isogas) {
    if (!c) return RTB_ERR_ARG;
    if (ntab <= 0 || !paths) return fail(c, RTB_ERR_ARG, "load_ktables: no files");
    std::vector<Kta> hd(ntab);
    std::vector<float> vmin(ntab), delv(ntab), data;
    std::vector<int> nbin(ntab);
    for (int t = 0; t < ntab; ++t) {
        File fl(paths[t]);
        if (!fl.f) return fail(c, RTB_ERR_ARG, "cannot open %s", paths[t] ? paths[t] : "(null)");
        std::string err;
        const int r = read_kta_header(fl.f, hd[t], err);
        if (r) return fail(c, r, "%s: %s", paths[t], err.c_str());
        const Kta& k = hd[t];
        // every table shares the /INTERPK/ grid of get_kg.f:100-101
        if (t > 0 && (k.np != hd[0].np || k.nt != hd[0].nt || k.ng != hd[0].ng || k.press != hd[0].press ||
                      k.temp != hd[0].temp || k.delg != hd[0].delg))
            return fail(c, RTB_ERR_UNSUPPORTED, "%s: P/T/g grid differs from %s", paths[t], paths[0]);
        const size_t n = (size_t)k.npoint * k.np * std::abs(k.nt) * k.ng;
        const size_t off = data.size();
        data.resize(off + n);
        if (!recs4(fl.f, k.irec0, n, data.data() + off))
            return fail(c, RTB_ERR_ARG, "%s: fewer k records than NPOINT x NP x NT x NG", paths[t]);
        vmin[t] = k.vmin;
        delv[t] = k.delv;
        nbin[t] = k.npoint;
        if (idgas) idgas[t] = k.idgas;
        if (isogas) isogas[t] = k.isogas;
    }
    const Kta& k0 = hd[0];
    // irregular grids: every table's centres those of the first within MAXDX = 1e-4 per cent (read_klist.f:160-176)
    for (int t = 1; t < ntab && !k0.vcen.empty(); ++t)
        for (size_t j = 0; j < hd[t].vcen.size() && j < k0.vcen.size(); ++j) {
            const float dx = 100.0f * std::fabs((hd[t].vcen[j] - k0.vcen[j]) / hd[t].vcen[j]);
            if (dx > 1e-4f) return fail(c, RTB_ERR_ARG, "%s: wave centre %zu differs from %s", paths[t], j + 1, paths[0]);
        }
    std::vector<float> lnp(k0.np);
    for (int i = 0; i < k0.np; ++i) lnp[i] = logf(k0.press[i]);   // PRESS(J) = LOG(PRESS(J)), read_khead.f:83
    int r = rtb_set_ktables(c, ntab, k0.np, k0.nt, k0.ng, lnp.data(), k0.temp.data(), k0.delg.data(), vmin.data(),
                            delv.data(), nbin.data(), data.data());
    if (r) return r;
    std::vector<int> ids(ntab), isos(ntab);
    for (int t = 0; t < ntab; ++t) {
        ids[t] = hd[t].idgas;
        isos[t] = hd[t].isogas;
    }
    r = rtb_set_ktable_ids(c, ntab, ids.data(), isos.data());
    if (r || k0.vcen.empty()) return r;
    return rtb_set_ktable_centres(c, k0.npoint, k0.vcen.data());
}

int rtb_load_cia(rtb_context* c, const char* path, float dnu) {
    if (!c) return RTB_ERR_ARG;
    File fl(path);
    if (!fl.f) return fail(c, RTB_ERR_ARG, "cannot open %s", path ? path : "(null)");
    const size_t nt = RTB_CIA_NUMT, nk = (size_t)RTB_CIA_NUMPAIRS * RTB_CIA_NUMT * RTB_CIA_NUMWN;
    double temps[RTB_CIA_NUMT];
    std::vector<float> kcia(nk);
    int32_t m1 = 0, m2 = 0, m3 = 0, m4 = 0;
    bool ok = std::fread(&m1, 4, 1, fl.f) == 1 && m1 == (int32_t)(nt * 8) && std::fread(temps, 8, nt, fl.f) == nt &&
              std::fread(&m2, 4, 1, fl.f) == 1 && m2 == m1;
    ok = ok && std::fread(&m3, 4, 1, fl.f) == 1 && m3 == (int32_t)(nk * 4) &&
         std::fread(kcia.data(), 4, nk, fl.f) == nk && std::fread(&m4, 4, 1, fl.f) == 1 && m4 == m3;
    if (!ok)
        return fail(c, RTB_ERR_ARG, "%s: not a CIA table (two unformatted records: 25 DOUBLE, REAL(9,25,1501))",
                    path);
    return rtb_set_cia(c, dnu, temps, kcia.data());
}

// the para-H2 CIA table (fpread_all.f:45-97): five sequential unformatted
// records, REAL TEMPK2(25), FP(IPARA), KH2H2(IPARA,25,1501),
// KH2HE(IPARA,25,1501), KCIA5(5,25,1501), each framed by 4-byte lengths
int rtb_load_para_cia(rtb_context* c, const char* path, float dnu2, int ipara) {
    if (!c) return RTB_ERR_ARG;
    if (ipara != 12 && ipara != 24) return fail(c, RTB_ERR_ARG, "para-H2 CIA: ipara %d (12 or 24)", ipara);
    File fl(path);
    if (!fl.f) return fail(c, RTB_ERR_ARG, "cannot open %s", path ? path : "(null)");
    const size_t nk = (size_t)ipara * RTB_CIA_NUMT * RTB_CIA_NUMWN, n5 = (size_t)5 * RTB_CIA_NUMT * RTB_CIA_NUMWN;
    std::vector<float> temps(RTB_CIA_NUMT), fp(ipara), kh2h2(nk), kh2he(nk), k5(n5);
    auto rec = [&](float* dst, size_t n) {
        int32_t m1 = 0, m2 = 0;
        return std::fread(&m1, 4, 1, fl.f) == 1 && m1 == (int32_t)(n * 4) && std::fread(dst, 4, n, fl.f) == n &&
               std::fread(&m2, 4, 1, fl.f) == 1 && m2 == m1;
    };
    if (!(rec(temps.data(), temps.size()) && rec(fp.data(), fp.size()) && rec(kh2h2.data(), nk) &&
          rec(kh2he.data(), nk) && rec(k5.data(), n5)))
        return fail(c, RTB_ERR_ARG, "%s: not a para-H2 CIA table of %d fractions (fpread_all.f:45-97)", path, ipara);
    return rtb_set_para_cia(c, dnu2, ipara, temps.data(), fp.data(), kh2h2.data(), kh2he.data(), k5.data());
}

// the stellar spectrum file of init_solar_wave.f:22-78: comment lines
// starting '#', the wavespace, the stellar radius, then records WAVE RAD up
// to the end of the file (at most MAXBIN = 16000, arrdef.f:19)
int rtb_load_stellar_spectrum(rtb_context* c, const char* path, int ispace) {
    if (!c) return RTB_ERR_ARG;
    File fl(path);
    if (!fl.f) return fail(c, RTB_ERR_ARG, "cannot open %s", path ? path : "(null)");
    char line[4096];
    std::string first;
    while (std::fgets(line, sizeof line, fl.f)) {
        if (line[0] == '#') continue;
        first = line;
        break;
    }
    int ispace1 = 0;
    {
        std::string tok;
        for (char ch : first) {
            if (ch == ' ' || ch == '\t' || ch == ',' || ch == '\n' || ch == '\r') {
                if (!tok.empty()) break;
            } else {
                tok += ch;
            }
        }
        if (!to_int(tok, ispace1)) return fail(c, RTB_ERR_ARG, "%s: no wavespace line", path);
    }
    if (ispace1 != ispace)
        return fail(c, RTB_ERR_ARG, "%s: wavespace %d of the stellar file is not the calculation's %d", path, ispace1,
                    ispace);
    std::vector<std::string> t;
    float solrad = 0.0f;
    if (!list_read(fl.f, 1, t) || !to_real(t[0], solrad)) return fail(c, RTB_ERR_ARG, "%s: no stellar radius", path);
    std::vector<float> wave, rad;
    constexpr int kMaxBin = 16000;
    while (list_read(fl.f, 2, t)) {
        float w, r;
        if (!to_real(t[0], w) || !to_real(t[1], r)) return fail(c, RTB_ERR_ARG, "%s: record %zu is not WAVE RAD", path,
                                                                wave.size() + 1);
        if ((int)wave.size() == kMaxBin) return fail(c, RTB_ERR_LIMIT, "%s: more than MAXBIN = %d points", path, kMaxBin);
        wave.push_back(w);
        rad.push_back(r);
    }
    return rtb_set_stellar_spectrum(c, (int)wave.size(), wave.data(), rad.data());
}

// e3tab.dat (e3interp.f:22-32): N, a header line, then N records TAU TRAN E3
int rtb_load_e3_table(rtb_context* c, const char* path) {
    if (!c) return RTB_ERR_ARG;
    File fl(path);
    if (!fl.f) return fail(c, RTB_ERR_ARG, "cannot open %s", path ? path : "(null)");
    std::vector<std::string> t;
    int n = 0;
    if (!list_read(fl.f, 1, t) || !to_int(t[0], n) || n <= 0 || n > 100000)
        return fail(c, RTB_ERR_ARG, "%s: no point count", path);
    char line[4096];
    if (!std::fgets(line, sizeof line, fl.f)) return fail(c, RTB_ERR_ARG, "%s: no header line", path);
    std::vector<double> tran(n), e3(n);
    for (int i = 0; i < n; ++i) {
        if (!list_read(fl.f, 3, t)) return fail(c, RTB_ERR_ARG, "%s: short table", path);
        for (std::string& x : t)
            for (char& ch : x)
                if (ch == 'd' || ch == 'D') ch = 'e';
        char *e1 = nullptr, *e2 = nullptr;
        tran[i] = std::strtod(t[1].c_str(), &e1);
        e3[i] = std::strtod(t[2].c_str(), &e2);
        if (*e1 || *e2) return fail(c, RTB_ERR_ARG, "%s: record %d is not TAU TRAN E3", path, i + 1);
    }
    return rtb_set_e3_table(c, n, tran.data(), e3.data());
}

// .fwh (cirsrtfg_wave.f:191-196): NFWHM, then NFWHM records VFWHM XFWHM
int rtb_read_fwh(const char* path, int* n, float* v, float* x, int cap) {
    File fl(path);
    if (!fl.f || !n) return RTB_ERR_ARG;
    std::vector<std::string> t;
    int m = 0;
    if (!list_read(fl.f, 1, t) || !to_int(t[0], m) || m < 0) return RTB_ERR_ARG;
    *n = m;
    if (!v && !x) return RTB_OK;
    if (!v || !x) return RTB_ERR_ARG;
    if (m > cap) return RTB_ERR_LIMIT;
    for (int i = 0; i < m; ++i)
        if (!list_read(fl.f, 2, t) || !to_real(t[0], v[i]) || !to_real(t[1], x[i])) return RTB_ERR_ARG;
    return RTB_OK;
}

// .fil (cirsconv.f:185-196): NCONV1, then per filter VCENTRAL, NSUB and NSUB
// records VFIL FIL
int rtb_read_fil(const char* path, int* nfil, int* npts, float* vcen, int* nsub, float* vfil, float* fil,
                 int cap_fil, int cap_pts) {
    File fl(path);
    if (!fl.f || !nfil || !npts) return RTB_ERR_ARG;
    std::vector<std::string> t;
    int m = 0;
    if (!list_read(fl.f, 1, t) || !to_int(t[0], m) || m < 0) return RTB_ERR_ARG;
    std::vector<float> vc(m), pv, pf;
    std::vector<int> ns(m);
    for (int k = 0; k < m; ++k) {
        if (!list_read(fl.f, 1, t) || !to_real(t[0], vc[k])) return RTB_ERR_ARG;
        if (!list_read(fl.f, 1, t) || !to_int(t[0], ns[k]) || ns[k] < 0) return RTB_ERR_ARG;
        for (int j = 0; j < ns[k]; ++j) {
            float a = 0.0f, b = 0.0f;
            if (!list_read(fl.f, 2, t) || !to_real(t[0], a) || !to_real(t[1], b)) return RTB_ERR_ARG;
            pv.push_back(a);
            pf.push_back(b);
        }
    }
    *nfil = m;
    *npts = (int)pv.size();
    if (!vcen && !nsub && !vfil && !fil) return RTB_OK;
    if (!vcen || !nsub || !vfil || !fil) return RTB_ERR_ARG;
    if (m > cap_fil || (int)pv.size() > cap_pts) return RTB_ERR_LIMIT;
    std::copy(vc.begin(), vc.end(), vcen);
    std::copy(ns.begin(), ns.end(), nsub);
    std::copy(pv.begin(), pv.end(), vfil);
    std::copy(pf.begin(), pf.end(), fil);
    return RTB_OK;
}

}  // extern "C"
