/* cirsrtfg_harness.c -- a plain C caller of the C ABI, the way a Fortran
 * program binds it: the /LAYCOM/, /PATHVA/ and /LGRAD/ arrays and xmap live in
 * static arrays with the reference's leading dimensions (MAXLAY, MAXINC,
 * MAXV, MAXGAS+2+MAXCON, MAXPRO; radtran/includes/arrdef.f,
 * pathcom.f) and rtb_cirsrtfg_wave receives them with ld_* = 0, the
 * reference defaults.  No Python is involved.
 *
 *   cirsrtfg_harness <inputs.bin> <outputs.bin>
 *
 * inputs.bin (little endian, every array preceded by nothing: sizes come
 * first): int32 ntab, np, nt, ng; float lnp[np], tk[|nt|], delg[ng],
 * vmin[ntab], delv[ntab]; int32 nbin[ntab]; float data[sum nbin*np*|nt|*ng];
 * float dnu; double temps[25]; float kcia[9*25*1501];
 * int32 nlayer, ngas, npath, npro, nv, nwave, nem, inormal, iray, itype,
 * ispace; float tsurf; float press, temp, delh [nlayer];
 * float pp, amount [ngas][nlayer]; int32 idgas, isogas, ktab [ngas];
 * int32 nlayin, imod [npath]; int32 layinc [npath][nlayer];
 * float scale, emtemp [npath][nlayer]; float dte, dam [npro][nlayer];
 * float xmap [npro][ngas+1][nv]; float vwave[nwave]; float vem, emis [nem].
 * outputs.bin: float calcout[npath*nwave], gradients[npath*nv*nwave],
 * gradtsurf[npath*nwave].
 * Exit status: 0 ok; 2 bad input file; 3 no CUDA device (the library
 * refuses to create a context, RTB_ERR_CUDA); 4 any other library error. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "radtran_b200.h"

#define NPARAM_MAX (RTB_MAXGAS + 2 + RTB_MAXCON)

/* Fortran-layout storage, as the COMMON blocks hold it */
static float press[RTB_MAXLAY], temp[RTB_MAXLAY], delh[RTB_MAXLAY];
static float pp[RTB_MAXGAS][RTB_MAXLAY], amount[RTB_MAXGAS][RTB_MAXLAY];
static int idgas[RTB_MAXGAS], isogas[RTB_MAXGAS], ktab[RTB_MAXGAS];
static int nlayin[RTB_MAXPAT], imod[RTB_MAXPAT], layinc[RTB_MAXPAT][RTB_MAXLAY];
static float scale[RTB_MAXPAT][RTB_MAXLAY], emtemp[RTB_MAXPAT][RTB_MAXLAY];
static float dte[RTB_MAXPRO][RTB_MAXLAY], dam[RTB_MAXPRO][RTB_MAXLAY];
static float xmap[RTB_MAXPRO][NPARAM_MAX][RTB_MAXV];

static FILE* fin;
static int rd(void* p, size_t size, size_t n) { return fread(p, size, n, fin) == n; }
static void* rd_new(size_t size, size_t n, int* ok) {
    void* p = malloc(size * (n ? n : 1));
    if (!p || !rd(p, size, n)) *ok = 0;
    return p;
}

int main(int argc, char** argv) {
    if (argc != 3) {
        fprintf(stderr, "usage: %s inputs.bin outputs.bin\n", argv[0]);
        return 2;
    }
    fin = fopen(argv[1], "rb");
    if (!fin) return 2;
    int ok = 1;
    int hdr[4];
    if (!rd(hdr, 4, 4)) return 2;
    const int ntab = hdr[0], np = hdr[1], nt = hdr[2], ng = hdr[3], ant = nt < 0 ? -nt : nt;
    float* lnp = rd_new(4, np, &ok);
    float* tk = rd_new(4, nt < 0 ? (size_t)np * ant : (size_t)ant, &ok);
    float* delg = rd_new(4, ng, &ok);
    float* vmin = rd_new(4, ntab, &ok);
    float* delv = rd_new(4, ntab, &ok);
    int* nbin = rd_new(4, ntab, &ok);
    if (!ok) return 2;
    size_t nrec = 0;
    for (int t = 0; t < ntab; ++t) nrec += (size_t)nbin[t];
    float* data = rd_new(4, nrec * np * ant * ng, &ok);
    float dnu;
    double temps[25];
    ok = ok && rd(&dnu, 4, 1) && rd(temps, 8, 25);
    float* kcia = rd_new(4, 9 * 25 * 1501, &ok);
    int s[11];
    float tsurf;
    ok = ok && rd(s, 4, 11) && rd(&tsurf, 4, 1);
    if (!ok) return 2;
    const int nlayer = s[0], ngas = s[1], npath = s[2], npro = s[3], nv = s[4], nwave = s[5], nem = s[6];
    if (nlayer > RTB_MAXLAY || ngas > RTB_MAXGAS || npath > RTB_MAXPAT || npro > RTB_MAXPRO || nv > RTB_MAXV)
        return 2;
    ok = rd(press, 4, nlayer) && rd(temp, 4, nlayer) && rd(delh, 4, nlayer);
    for (int g = 0; g < ngas && ok; ++g) ok = rd(pp[g], 4, nlayer);
    for (int g = 0; g < ngas && ok; ++g) ok = rd(amount[g], 4, nlayer);
    ok = ok && rd(idgas, 4, ngas) && rd(isogas, 4, ngas) && rd(ktab, 4, ngas);
    ok = ok && rd(nlayin, 4, npath) && rd(imod, 4, npath);
    for (int p = 0; p < npath && ok; ++p) ok = rd(layinc[p], 4, nlayer);
    for (int p = 0; p < npath && ok; ++p) ok = rd(scale[p], 4, nlayer);
    for (int p = 0; p < npath && ok; ++p) ok = rd(emtemp[p], 4, nlayer);
    for (int k = 0; k < npro && ok; ++k) ok = rd(dte[k], 4, nlayer);
    for (int k = 0; k < npro && ok; ++k) ok = rd(dam[k], 4, nlayer);
    for (int k = 0; k < npro && ok; ++k)
        for (int q = 0; q <= ngas && ok; ++q) ok = rd(xmap[k][q], 4, nv);
    float* vwave = rd_new(4, nwave, &ok);
    float* vem = rd_new(4, nem, &ok);
    float* emis = rd_new(4, nem, &ok);
    fclose(fin);
    if (!ok) return 2;

    rtb_context* ctx = NULL;
    int st = rtb_create(0, &ctx);
    if (st != RTB_OK) {
        fprintf(stderr, "rtb_create: status %d\n", st);
        return st == RTB_ERR_CUDA ? 3 : 4;
    }
    st = rtb_set_ktables(ctx, ntab, np, nt, ng, lnp, tk, delg, vmin, delv, nbin, data);
    if (st == RTB_OK) st = rtb_set_cia(ctx, dnu, temps, kcia);
    rtb_atm a;
    memset(&a, 0, sizeof a);               /* ld_* = 0: MAXLAY, MAXCON, MAXV, MAXGAS+2+MAXCON */
    a.nlayer = nlayer; a.ngas = ngas; a.ncont = 0; a.npath = npath; a.npro = npro; a.nv = nv; a.nwave = nwave;
    a.press = press; a.temp = temp; a.delh = delh;
    a.pp = &pp[0][0]; a.amount = &amount[0][0];
    a.idgas = idgas; a.isogas = isogas; a.ktab = ktab;
    a.nlayin = nlayin; a.imod = imod; a.layinc = &layinc[0][0];
    a.scale = &scale[0][0]; a.emtemp = &emtemp[0][0];
    a.dte = &dte[0][0]; a.dam = &dam[0][0];
    a.xmap = &xmap[0][0][0];
    a.vwave = vwave;
    a.inormal = s[7]; a.iray = s[8]; a.itype = s[9]; a.ispace = s[10];
    a.tsurf = tsurf;
    a.nem = nem; a.vem = vem; a.emissivity = emis;
    const size_t n1 = (size_t)npath * nwave, n2 = n1 * nv;
    float* calcout = calloc(n1, 4);
    float* gradients = calloc(n2 ? n2 : 1, 4);
    float* gradtsurf = calloc(n1, 4);
    if (st == RTB_OK) st = rtb_cirsrtfg_wave(ctx, &a, calcout, gradients, gradtsurf);
    if (st != RTB_OK) {
        fprintf(stderr, "status %d: %s\n", st, rtb_last_error(ctx));
        rtb_destroy(ctx);
        return 4;
    }
    rtb_destroy(ctx);
    FILE* fo = fopen(argv[2], "wb");
    if (!fo) return 2;
    ok = fwrite(calcout, 4, n1, fo) == n1 && fwrite(gradients, 4, n2, fo) == n2 && fwrite(gradtsurf, 4, n1, fo) == n1;
    fclose(fo);
    return ok ? 0 : 2;
}
