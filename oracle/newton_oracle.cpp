/*
 * newton_oracle.cpp -- ORACLE (test infrastructure only; see oracle.h).
 *
 * Restatement of the optimal-estimation Newton step of the reference:
 *   nemesis/calc_gain_matrix.f:70-163   gain matrix and averaging kernels
 *   radtran/matrices/dinvertm.f:114-170 Cholesky inverse + A*Ainv check
 *   radtran/matrices/dcholdc.f:62-92, dcholsl.f:46-59
 *   radtran/matrices/dmult_mat.f:49-57  C = A*B (k outer, i, s inner)
 *   nemesis/calcnextxn.f:64-104         x_out = x0 + D(y-yn) - AA(x0-xn)
 *   nemesis/calc_phiret.f:49-102        phi = chi2 + prior term
 * All arithmetic is DOUBLE PRECISION as in the reference; REAL inputs are
 * promoted exactly where the reference promotes them.
 */
#include "oracle.h"

#include <cmath>
#include <cstring>
#include <vector>

namespace {

/* dmult_mat.f:49-57 on column-major arrays with explicit leading dims */
void dmult(const double* a, int lda, int a1, int a2, const double* b, int ldb, int b2, double* c, int ldc) {
    for (int k = 0; k < b2; ++k)
        for (int i = 0; i < a1; ++i) {
            double cik = 0.0;
            for (int s = 0; s < a2; ++s) cik = cik + a[i + (size_t)lda * s] * b[s + (size_t)ldb * k];
            c[i + (size_t)ldc * k] = cik;
        }
}

/* dcholdc.f:62-92.  a: (n, n) lda; upper triangle in, factor L below. */
void dcholdc(double* a, int n, int lda, double* p, bool* nonpd) {
    for (int i = 0; i < n; ++i)
        for (int j = i; j < n; ++j) {
            double sum = a[i + (size_t)lda * j];
            for (int k = i - 1; k >= 0; --k) sum = sum - a[i + (size_t)lda * k] * a[j + (size_t)lda * k];
            if (i == j) {
                if (sum <= 0.) { p[i] = 1.0; if (nonpd) *nonpd = true; }
                else p[i] = std::sqrt(sum);
            } else {
                a[j + (size_t)lda * i] = sum / p[i];
            }
        }
}

/* dcholsl.f:46-59 */
void dcholsl(const double* a, int n, int lda, const double* p, const double* b, double* x) {
    for (int i = 0; i < n; ++i) {
        double sum = b[i];
        for (int k = i - 1; k >= 0; --k) sum = sum - a[i + (size_t)lda * k] * x[k];
        x[i] = sum / p[i];
    }
    for (int i = n - 1; i >= 0; --i) {
        double sum = x[i];
        for (int k = i + 1; k < n; ++k) sum = sum - a[k + (size_t)lda * i] * x[k];
        x[i] = sum / p[i];
    }
}

/* dinvertm.f jmod = 2 (:114-141) and the inversion check (:145-170). */
int dinvertm_chol(int n, int lda, const double* A, double* ainv, int ldi) {
    std::vector<double> A1((size_t)n * n, 0.0), P(n), B1(n), X(n);
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i < j; ++i) ainv[i + (size_t)ldi * j] = 0.0;
        for (int i = j; i < n; ++i) {
            A1[j + (size_t)n * i] = A[j + (size_t)lda * i];
            ainv[i + (size_t)ldi * j] = 0.0;
        }
        ainv[j + (size_t)ldi * j] = 1.0;
    }
    dcholdc(A1.data(), n, n, P.data(), nullptr);
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i < n; ++i) B1[i] = ainv[i + (size_t)ldi * j];
        dcholsl(A1.data(), n, n, P.data(), B1.data(), X.data());
        for (int i = 0; i < n; ++i) ainv[i + (size_t)ldi * j] = X[i];
    }
    int icheck = 0;
    std::vector<double> Ac((size_t)n * n), Ai((size_t)n * n), IDE((size_t)n * n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            Ac[i + (size_t)n * j] = A[i + (size_t)lda * j];
            Ai[i + (size_t)n * j] = ainv[i + (size_t)ldi * j];
            if (std::isnan(Ai[i + (size_t)n * j])) icheck = 1;
        }
    dmult(Ac.data(), n, n, n, Ai.data(), n, n, IDE.data(), n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            const double dx = (i == j) ? std::fabs(1.0 - IDE[i + (size_t)n * j]) : std::fabs(IDE[i + (size_t)n * j]);
            if (dx > 1e-3) icheck = 1;   /* TINY = 1E-3 (REAL literal) */
        }
    return icheck;
}

}  // namespace

extern "C" {

int orc_dinvertm_chol(int n, int lda, const double* a, double* ainv) {
    return dinvertm_chol(n, lda, a, ainv, lda);
}

int orc_calc_gain_matrix(int nx, int ny, int ldx, int ldy, const float* kk_in, const float* sx_in,
                         const double* sxi, const float* se_in, const double* sei, double* dd_out,
                         double* aa_out, int* icheck) {
    const int n1 = nx, n2 = ny;
    std::vector<double> kk((size_t)ny * nx), kt((size_t)nx * ny);
    for (int i = 0; i < ny; ++i)
        for (int j = 0; j < nx; ++j) {
            const double v = (double)kk_in[i + (size_t)ldy * j];
            kk[i + (size_t)ny * j] = v;
            kt[j + (size_t)nx * i] = v;
        }
    std::vector<double> dd((size_t)nx * ny), a;
    int ic = 0;
    if (nx >= ny) {                                        /* calc_gain_matrix.f:86-121 */
        std::vector<double> sx((size_t)nx * nx), m((size_t)nx * ny), aa((size_t)ny * ny), b((size_t)ny * ny);
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < nx; ++j) sx[i + (size_t)nx * j] = (double)sx_in[i + (size_t)ldx * j];
        dmult(sx.data(), nx, nx, nx, kt.data(), nx, ny, m.data(), nx);
        dmult(kk.data(), ny, ny, nx, m.data(), nx, ny, aa.data(), ny);
        for (int i = 0; i < ny; ++i)
            for (int j = 0; j < ny; ++j) aa[i + (size_t)ny * j] = aa[i + (size_t)ny * j] + (double)se_in[i + (size_t)ldy * j];
        ic = dinvertm_chol(ny, ny, aa.data(), b.data(), ny);
        dmult(m.data(), nx, nx, ny, b.data(), ny, ny, dd.data(), nx);
    } else {                                               /* :123-149 */
        std::vector<double> se((size_t)ny * ny), m((size_t)nx * ny), c((size_t)nx * nx), ai((size_t)nx * nx);
        for (int i = 0; i < ny; ++i)
            for (int j = 0; j < ny; ++j) se[i + (size_t)ny * j] = sei[i + (size_t)ldy * j];
        dmult(kt.data(), nx, nx, ny, se.data(), ny, ny, m.data(), nx);
        dmult(m.data(), nx, nx, ny, kk.data(), ny, nx, c.data(), nx);
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < nx; ++j) c[j + (size_t)nx * i] = c[j + (size_t)nx * i] + sxi[j + (size_t)ldx * i];
        ic = dinvertm_chol(nx, nx, c.data(), ai.data(), nx);
        dmult(ai.data(), nx, nx, nx, m.data(), nx, ny, dd.data(), nx);
    }
    std::vector<double> aa((size_t)nx * nx);
    dmult(dd.data(), nx, nx, ny, kk.data(), ny, nx, aa.data(), nx);
    for (int i = 0; i < nx; ++i) {
        for (int j = 0; j < ny; ++j) dd_out[i + (size_t)ldx * j] = dd[i + (size_t)nx * j];
        for (int j = 0; j < nx; ++j) aa_out[i + (size_t)ldx * j] = aa[i + (size_t)nx * j];
    }
    (void)n1; (void)n2;
    if (icheck) *icheck = ic;
    return RTB_OK;
}

int orc_calc_gain_matrix_diag(int nx, int ny, int ldx, int ldy, const float* kk_in, const double* sxi,
                              const double* sei_diag, double* dd_out, double* aa_out, int* icheck) {
    if (!(nx < ny)) return RTB_ERR_UNSUPPORTED;
    std::vector<double> kk((size_t)ny * nx), m((size_t)nx * ny), c((size_t)nx * nx), ai((size_t)nx * nx),
        dd((size_t)nx * ny), aa((size_t)nx * nx);
    for (int i = 0; i < ny; ++i)
        for (int j = 0; j < nx; ++j) kk[i + (size_t)ny * j] = (double)kk_in[i + (size_t)ldy * j];
    /* m = kt*sei with diagonal sei: every off-diagonal product is an exact
     * zero, so m(i,k) = kk(k,i)*sei(k,k) bit-for-bit as in the dense loop */
    for (int k = 0; k < ny; ++k)
        for (int i = 0; i < nx; ++i) m[i + (size_t)nx * k] = kk[k + (size_t)ny * i] * sei_diag[k];
    dmult(m.data(), nx, nx, ny, kk.data(), ny, nx, c.data(), nx);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < nx; ++j) c[j + (size_t)nx * i] = c[j + (size_t)nx * i] + sxi[j + (size_t)ldx * i];
    const int ic = dinvertm_chol(nx, nx, c.data(), ai.data(), nx);
    dmult(ai.data(), nx, nx, nx, m.data(), nx, ny, dd.data(), nx);
    dmult(dd.data(), nx, nx, ny, kk.data(), ny, nx, aa.data(), nx);
    for (int i = 0; i < nx; ++i) {
        for (int j = 0; j < ny; ++j) dd_out[i + (size_t)ldx * j] = dd[i + (size_t)nx * j];
        for (int j = 0; j < nx; ++j) aa_out[i + (size_t)ldx * j] = aa[i + (size_t)nx * j];
    }
    if (icheck) *icheck = ic;
    return RTB_OK;
}

void orc_calcnextxn(int nx, int ny, int ldx, const float* x0, const float* xn, const float* y, const float* yn,
                    const double* dd, const double* aa, float* x_out) {
    std::vector<double> b(nx), c(ny), x1(nx), x2(nx);
    for (int i = 0; i < nx; ++i) b[i] = (double)(x0[i] - xn[i]);
    for (int i = 0; i < nx; ++i) {
        double s = 0.0;
        for (int k = 0; k < nx; ++k) s = s + aa[i + (size_t)ldx * k] * b[k];
        x1[i] = s;
    }
    for (int i = 0; i < ny; ++i) c[i] = (double)(y[i] - yn[i]);
    for (int i = 0; i < nx; ++i) {
        double s = 0.0;
        for (int k = 0; k < ny; ++k) s = s + dd[i + (size_t)ldx * k] * c[k];
        x2[i] = s;
    }
    for (int i = 0; i < nx; ++i) x_out[i] = x0[i] + (float)(x2[i] - x1[i]);
}

/* calc_serr.f (sm = dd se dd^T, sn = (aa - I) sx (aa - I)^T, st = sn + sm),
 * diagonal se; REAL outputs (ldx, nx). */
void orc_calc_serr_diag(int nx, int ny, int ldx, const float* sx_in, const float* se_diag, const double* dd_in,
                        const double* aa_in, float* st_out, float* sn_out, float* sm_out) {
    std::vector<double> a((size_t)nx * ny), dt((size_t)ny * nx), sm((size_t)nx * nx), b((size_t)nx * nx),
        e((size_t)nx * nx), c((size_t)nx * nx), sn((size_t)nx * nx);
    /* a = dd*se: the off-diagonal products of the dense se are exact zeros */
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            a[i + (size_t)nx * j] = dd_in[i + (size_t)ldx * j] * (double)se_diag[j];
            dt[j + (size_t)ny * i] = dd_in[i + (size_t)ldx * j];
        }
    dmult(a.data(), nx, nx, ny, dt.data(), ny, nx, sm.data(), nx);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < nx; ++j) {
            b[i + (size_t)nx * j] = (double)sx_in[i + (size_t)ldx * j];
            e[i + (size_t)nx * j] = aa_in[i + (size_t)ldx * j];
        }
    for (int i = 0; i < nx; ++i) e[i + (size_t)nx * i] = e[i + (size_t)nx * i] - 1.0;
    dmult(e.data(), nx, nx, nx, b.data(), nx, nx, c.data(), nx);
    std::vector<double> et((size_t)nx * nx);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < nx; ++j) et[i + (size_t)nx * j] = e[j + (size_t)nx * i];
    dmult(c.data(), nx, nx, nx, et.data(), nx, nx, sn.data(), nx);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < nx; ++j) {
            const size_t k = i + (size_t)nx * j, o = i + (size_t)ldx * j;
            sm_out[o] = (float)sm[k];
            sn_out[o] = (float)sn[k];
            st_out[o] = (float)(sm[k] + sn[k]);
        }
}
float orc_calc_phiret(int ny, int ldy, const float* y, const float* yn, const double* sei, int nx, int ldx,
                      const float* xn, const float* xa, const double* sai, float* chisq) {
    std::vector<double> b(ny), a(ny);
    for (int i = 0; i < ny; ++i) b[i] = (double)(yn[i] - y[i]);
    for (int i = 0; i < ny; ++i) {
        double s = 0.0;
        for (int k = 0; k < ny; ++k) s = s + sei[i + (size_t)ldy * k] * b[k];
        a[i] = s;
    }
    double phi1 = 0.0;
    for (int k = 0; k < ny; ++k) phi1 = phi1 + b[k] * a[k];
    if (chisq) *chisq = (float)phi1;
    std::vector<double> bx(nx), ax(nx);
    for (int i = 0; i < nx; ++i) bx[i] = (double)(xn[i] - xa[i]);
    for (int i = 0; i < nx; ++i) {
        double s = 0.0;
        for (int k = 0; k < nx; ++k) s = s + sai[i + (size_t)ldx * k] * bx[k];
        ax[i] = s;
    }
    double phi2 = 0.0;
    for (int k = 0; k < nx; ++k) phi2 = phi2 + bx[k] * ax[k];
    return (float)(phi1 + phi2);
}

float orc_calc_phiret_diag(int ny, const float* y, const float* yn, const double* sei_diag, int nx, int ldx,
                           const float* xn, const float* xa, const double* sai, float* chisq) {
    double phi1 = 0.0;
    for (int k = 0; k < ny; ++k) {
        const double b = (double)(yn[k] - y[k]);
        phi1 = phi1 + b * (sei_diag[k] * b);
    }
    if (chisq) *chisq = (float)phi1;
    std::vector<double> bx(nx), ax(nx);
    for (int i = 0; i < nx; ++i) bx[i] = (double)(xn[i] - xa[i]);
    for (int i = 0; i < nx; ++i) {
        double s = 0.0;
        for (int k = 0; k < nx; ++k) s = s + sai[i + (size_t)ldx * k] * bx[k];
        ax[i] = s;
    }
    double phi2 = 0.0;
    for (int k = 0; k < nx; ++k) phi2 = phi2 + bx[k] * ax[k];
    return (float)(phi1 + phi2);
}

}  // extern "C"

/* ---- instrument convolution (radtran/cirsrad/cirsconv.f:12-246: FWHM > 0
 * with an optional .fwh width table, FWHM = 0, FWHM < 0 filter channels) with CSPLINE (rtm_util/cspline.f) and CSPLINT
 * (rtm_util/csplint.f); REAL arithmetic as the reference, DOUBLE sums. ---- */
namespace {
void cspline_nat(const float* X, const float* Y, int N, float* Y2, std::vector<float>& U) {
    U.assign(N, 0.0f);
    Y2[0] = 0.0f;                                   /* YP1 > .99E30: natural */
    U[0] = 0.0f;
    for (int I = 1; I < N - 1; ++I) {
        const float SIG = (X[I] - X[I - 1]) / (X[I + 1] - X[I - 1]);
        const float P = SIG * Y2[I - 1] + 2.0f;
        Y2[I] = (SIG - 1.0f) / P;
        if (X[I - 1] == X[I] || X[I] == X[I + 1]) {
            U[I] = U[I - 1];
            continue;
        }
        U[I] = (6.0f * ((Y[I + 1] - Y[I]) / (X[I + 1] - X[I]) - (Y[I] - Y[I - 1]) / (X[I] - X[I - 1])) /
                    (X[I + 1] - X[I - 1]) - SIG * U[I - 1]) / P;
    }
    const float QN = 0.0f, UN = 0.0f;              /* YPN > .99E30 */
    Y2[N - 1] = (UN - QN * U[N - 2]) / (QN * Y2[N - 2] + 1.0f);
    for (int K = N - 2; K >= 0; --K) Y2[K] = Y2[K] * Y2[K + 1] + U[K];
}

float csplint(const float* XA, const float* YA, const float* Y2A, int N, float X) {
    int KLO = 1, KHI = N;
    while (KHI - KLO > 1) {
        const int K = (KHI + KLO) / 2;
        if (XA[K - 1] > X) KHI = K; else KLO = K;
    }
    const double H = (double)(XA[KHI - 1] - XA[KLO - 1]);
    const double A = (double)(XA[KHI - 1] - X) / H;
    const double B = (double)(X - XA[KLO - 1]) / H;
    const double Y1 = A * (double)YA[KLO - 1] + B * (double)YA[KHI - 1] +
                      ((A * A * A - A) * (double)Y2A[KLO - 1] + (B * B * B - B) * (double)Y2A[KHI - 1]) * (H * H) /
                          6.0;
    return std::fabs(Y1) > 1.00E-37 ? (float)Y1 : 1.00E-37f;
}
}  // namespace

namespace {
/* INTERP (rtm_util/interp.f:24-37); with verint, VERINT (radtran/path/verint.f:29-46) */
float interp_f(const float* X, const float* Y, int N, float XIN, bool verint) {
    int I = N;
    if (X[0] < X[N - 1]) {
        for (int k = 1; k <= N; ++k)
            if (X[k - 1] > XIN) { I = k; break; }
    } else {
        for (int k = 1; k <= N; ++k)
            if (X[k - 1] < XIN) { I = k; break; }
    }
    if (I == 1) I = 2;
    float YOUT = Y[I - 2] + (Y[I - 1] - Y[I - 2]) * (XIN - X[I - 2]) / (X[I - 1] - X[I - 2]);
    if (verint) {
        if (X[I - 2] == X[I - 1]) YOUT = Y[I - 1];
        if (std::isnan(YOUT)) YOUT = Y[I - 1];
    }
    return YOUT;
}
}  // namespace

extern "C" int orc_cirsconv_ex(float fwhm, int nwave, const float* vwave, const float* y, int nconv,
                               const float* vconv, int nfwhm, const float* vfwhm, const float* xfwhm, int nfil,
                               const float* vcen, const int* nsub, const float* vfil, const float* fil,
                               float* yout) {
    if (nwave == 1 && fwhm != 0.0f) {          /* cirsconv.f:45-54 */
        if (nconv != 1) return RTB_ERR_ARG;
        yout[0] = 1.0f;
        return RTB_OK;
    }
    if (fwhm == 0.0f) {                        /* cirsconv.f:162-169 */
        for (int i = 0; i < nconv; ++i) yout[i] = y[i];
        return RTB_OK;
    }
    if (fwhm < 0.0f) {                         /* cirsconv.f:171-239 */
        int off = 0;
        std::vector<float> ytmp(nwave);
        for (int k = 0; k < nfil; ++k) {
            const float* VF = vfil + off;
            const float* FF = fil + off;
            const int ns = nsub[k];
            off += ns;
            for (int i = 0; i < nconv; ++i) {
                const float dv = std::fabs(vcen[k] - vconv[i]);
                if (!(dv < 0.00001f)) continue;
                for (int j = 0; j < nwave; ++j)
                    ytmp[j] = (vwave[j] >= VF[0] && vwave[j] <= VF[ns - 1]) ? interp_f(VF, FF, ns, vwave[j], false)
                                                                             : 0.0f;
                double sumf = 0.0, sum = 0.0;
                for (int j = 0; j < nwave - 1; ++j)
                    if (ytmp[j] != 0.0f) {
                        const float delv = vwave[j + 1] - vwave[j];
                        const float a = ytmp[j] * y[j] * delv;
                        const float b = ytmp[j] * delv;
                        sum = sum + (double)a;
                        sumf = sumf + (double)b;
                    }
                yout[i] = (float)(sum / sumf);
            }
        }
        return RTB_OK;
    }
    std::vector<float> xc(vwave, vwave + nwave), yc(y, y + nwave);
    if (vconv[nconv - 1] > vwave[nwave - 1] - fwhm / 2.0f) {
        const float x = vconv[nconv - 1] + fwhm;
        xc.push_back(x);
        yc.push_back(y[nwave - 1] + ((y[nwave - 1] - y[nwave - 2]) / (vwave[nwave - 1] - vwave[nwave - 2]) *
                                     (x - vwave[nwave - 1])));
    }
    if (vconv[0] < vwave[0] + fwhm / 2.0f) {
        const float x = vconv[0] - fwhm;
        xc.insert(xc.begin(), x);
        yc.insert(yc.begin(), y[0] + ((y[1] - y[0]) / (vwave[1] - vwave[0]) * (x - vwave[0])));
    }
    std::vector<float> x1v, y1v;
    for (size_t i = 0; i < xc.size(); ++i)
        if (!std::isnan(yc[i])) {
            x1v.push_back(xc[i]);
            y1v.push_back(yc[i]);
        }
    const int nc = (int)x1v.size();
    std::vector<float> y2(nc), u;
    cspline_nat(x1v.data(), y1v.data(), nc, y2.data(), u);
    const int nstep = 20;
    for (int i = 0; i < nconv; ++i) {
        float yfwhm = fwhm;                    /* cirsconv.f:147-150 */
        if (nfwhm > 0) yfwhm = interp_f(vfwhm, xfwhm, nfwhm, vconv[i], true);
        const float x1 = vconv[i] - yfwhm / 2.0f, x2 = vconv[i] + yfwhm / 2.0f;
        const float delx = (x2 - x1) / (float)(nstep - 1);
        double sum = 0.0, yold = 0.0;
        for (int j = 1; j <= nstep; ++j) {
            const float xi = x1 + (float)(j - 1) * delx;
            const double yi = (double)csplint(x1v.data(), y1v.data(), y2.data(), nc, xi);
            if (j == 1) sum = 0.0;
            else sum = sum + (yi + yold) * (double)(delx / 2.0f);
            yold = yi;
        }
        yout[i] = (float)(sum / (double)fwhm);
    }
    return RTB_OK;
}

extern "C" int orc_cirsconv(int nwave, const float* vwave, const float* y, float fwhm, int nconv,
                            const float* vconv, float* yout) {
    if (fwhm < 0.0f || (fwhm > 0.0f && nwave < 2)) return RTB_ERR_UNSUPPORTED;
    return orc_cirsconv_ex(fwhm, nwave, vwave, y, nconv, vconv, 0, nullptr, nullptr, 0, nullptr, nullptr, nullptr,
                           nullptr, yout);
}
