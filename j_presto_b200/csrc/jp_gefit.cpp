// jp_gefit.cpp -- one McMD weight iteration on the host: from the energy histogram of a
// multicanonical run and the weight it ran with, the new d lnN/dE polynomial (.nf).
//
// Restates GEprep (src_GEprep/):
//   distrib_MULT.f90:60-68     bin layout: nAB = nBIN + 2 nBOR bins of width (maxE-minE)/nBIN
//                               starting nBOR bins below minE, centre EE(i)
//   distrib_MULT.f90:286-296   lnP = ln P - ln max P (empty bins marked)
//   distrib_MULT.f90:322-376   dlnN(i) = (lnP(i+1) - lnP(i))/dE + d lnN_old/dE at the upper
//                               edge of bin i (old polynomial, or alphalw/alphaup outside)
//   distrib_MULT.f90:386-445   data selection and weights sqrt(P(i)+P(i+1)), the fit on
//                               the next range [nxminE, nxmaxE], end values and .nf fields
//   lstsquare_final.f90        weighted windowed polynomial least squares: the window with
//                               the most weight fitted freely, the windows above it with C0/C1
//                               continuity imposed, the windows below it with C0/C1 continuity
//                               as Lagrange constraints; residual errors
//   minver.f90                 Gauss-Jordan inverse with partial pivoting (pivots below 1e-12
//                               zero their row and column)
// The run-weight (fw) and flatness-acceleration options of distrib_MULT are not restated:
// every histogram count has weight 1.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "jpgpu.h"

namespace {

double ipow(double x, int j) {
  double r = 1.0;
  for (int k = 0; k < j; ++k) r *= x;
  return r;
}

// minver.f90: in-place inverse of the m x m matrix a (row-major, leading dimension m)
void minver(std::vector<double>& a, int m) {
  const double eps = 1.0e-12;
  std::vector<int> iw(m);
  for (int i = 0; i < m; ++i) iw[i] = i;
  auto A = [&](int i, int j) -> double& { return a[(size_t)i * m + j]; };
  for (int k = 0; k < m; ++k) {
    double wmax = 0.0;
    int lr = k;
    for (int i = k; i < m; ++i) {
      const double w = std::fabs(A(i, k));
      if (w > wmax) { wmax = w; lr = i; }
    }
    const double pivot = A(lr, k), api = std::fabs(pivot);
    if (lr != k) {
      std::swap(iw[k], iw[lr]);
      for (int j = 0; j < m; ++j) std::swap(A(k, j), A(lr, j));
    }
    if (api > eps) {
      for (int j = 0; j < m; ++j) A(k, j) /= pivot;
      for (int i = 0; i < m; ++i) {
        if (i == k) continue;
        const double w = A(i, k);
        if (w != 0.0) {
          for (int j = 0; j < m; ++j)
            if (j != k) A(i, j) -= w * A(k, j);
          A(i, k) = -w / pivot;
        }
      }
      A(k, k) = 1.0 / pivot;
    } else {
      for (int j = 0; j < m; ++j) { A(k, j) = 0.0; A(j, k) = 0.0; }
    }
  }
  for (int i = 0; i < m; ++i) {
    while (iw[i] != i) {
      const int k = iw[i];
      std::swap(iw[k], iw[i]);
      for (int j = 0; j < m; ++j) std::swap(A(j, i), A(j, k));
    }
  }
}

// weighted power sums of one window's data range [imn, imx] (0-based, inclusive)
void power_sums(const double* X, const double* Y, const double* w, int imn, int imx, double x0,
                int ndim, std::vector<double>& xs, std::vector<double>& xys, double& swei) {
  xs.assign(2 * ndim + 1, 0.0);
  xys.assign(ndim + 1, 0.0);
  double sw = 0.0;
  for (int i = imn; i <= imx; ++i) sw += w[i];
  swei = 1.0 / sw;
  for (int i = imn; i <= imx; ++i) {
    const double dx = X[i] - x0;
    for (int j = 1; j <= 2 * ndim; ++j) xs[j] += ipow(dx, j) * w[i];
    for (int j = 0; j <= ndim; ++j) xys[j] += Y[i] * ipow(dx, j) * w[i];
  }
  for (int j = 1; j <= 2 * ndim; ++j) xs[j] *= swei;
  for (int j = 0; j <= ndim; ++j) xys[j] *= swei;
}

}  // namespace

extern "C" int jp_lstsq_windows(int32_t nwindow, int32_t ndat, int32_t ndim, double minv,
                                double maxv, const double *X, const double *Y, const double *wei,
                                double *coe, double *low, double *high, double *resid) {
  if (nwindow < 1 || ndim < 1 || ndat < 1 || !X || !Y || !wei || !coe || !low || !high)
    return JP_E_INVALID;
  const int nw = nwindow, nd = ndim;
  auto C = [&](int j, int w) -> double& { return coe[(size_t)w * (nd + 1) + j]; };
  for (int w = 0; w < nw; ++w)
    for (int j = 0; j <= nd; ++j) C(j, w) = 0.0;
  // window boundaries on the data (lstsquare_final.f90:37-51); nmx[w] = last data index
  std::vector<int> nmx(nw, ndat - 1);
  const double rr = (maxv - minv) / nw;
  double edge = rr + minv;
  const double tol = rr * 0.00001;
  int j = 0;
  low[0] = minv;
  for (int i = 0; i < ndat; ++i) {
    if (edge - X[i] < tol) {
      high[j] = X[i];
      nmx[j] = i;
      ++j;
      edge = rr * (j + 1) + minv;
      if (j == nw) break;
      low[j] = X[i];
    }
  }
  high[nw - 1] = maxv;
  nmx[nw - 1] = ndat - 1;
  const int itole = ndat / (2 * nw);
  // the window holding the most weight (:56-67)
  std::vector<double> nwin(nw, 0.0);
  int k0 = 0;
  for (int w = 0; w < nw; ++w) {
    for (int i = k0; i <= nmx[w]; ++i) nwin[w] += wei[i] * wei[i];
    k0 = nmx[w] + 1;
  }
  int maxw = 0;
  for (int w = 1; w < nw; ++w)
    if (nwin[w] > nwin[maxw]) maxw = w;
  std::vector<double> xs, xys;
  double swei;
  // free fit of that window (:69-101)
  {
    const int ii = maxw != 0 ? nmx[maxw - 1] : 0;
    const int imn = std::max(0, ii - itole), imx = std::min(nmx[maxw] + itole, ndat - 1);
    power_sums(X, Y, wei, imn, imx, low[maxw], nd, xs, xys, swei);
    std::vector<double> A((size_t)nd * nd), B(nd), Cc(nd);
    for (int a = 0; a < nd; ++a) {
      for (int b = 0; b < nd; ++b) A[(size_t)a * nd + b] = xs[a + b + 2] - xs[a + 1] * xs[b + 1];
      B[a] = xys[a + 1] - xys[0] * xs[a + 1];
    }
    minver(A, nd);
    for (int a = 0; a < nd; ++a) {
      double s = 0.0;
      for (int b = 0; b < nd; ++b) s += A[(size_t)a * nd + b] * B[b];
      Cc[a] = s;
    }
    double dot = 0.0;
    for (int a = 0; a < nd; ++a) dot += Cc[a] * xs[a + 1];
    C(0, maxw) = -dot + xys[0];
    for (int a = 0; a < nd; ++a) C(a + 1, maxw) = Cc[a];
  }
  // windows above: value and slope continuous at the lower edge (:105-142)
  for (int w = maxw + 1; w < nw; ++w) {
    const int p = w - 1;
    const double dx = high[p] - low[p];
    C(0, w) = C(0, p);
    for (int a = 1; a <= nd; ++a) C(0, w) += C(a, p) * ipow(dx, a);
    C(1, w) = C(1, p);
    for (int a = 2; a <= nd; ++a) C(1, w) += a * C(a, p) * ipow(dx, a - 1);
    const int imn = std::max(0, nmx[w - 1] - itole), imx = std::min(nmx[w] + itole, ndat - 1);
    power_sums(X, Y, wei, imn, imx, low[w], nd, xs, xys, swei);
    const int m = nd - 1;
    if (m >= 1) {
      std::vector<double> A((size_t)m * m), B(m);
      for (int a = 2; a <= nd; ++a) {
        for (int b = 2; b <= nd; ++b) A[(size_t)(a - 2) * m + (b - 2)] = xs[a + b];
        B[a - 2] = xys[a] - C(0, w) * xs[a] - C(1, w) * xs[a + 1];
      }
      minver(A, m);
      for (int a = 0; a < m; ++a) {
        double s = 0.0;
        for (int b = 0; b < m; ++b) s += A[(size_t)a * m + b] * B[b];
        C(a + 2, w) = s;
      }
    }
  }
  // windows below: continuity with the window above as two Lagrange constraints (:145-192)
  for (int w = maxw - 1; w >= 0; --w) {
    const int ii = w != 0 ? nmx[w - 1] : 0;
    const int imn = std::max(0, ii - itole), imx = std::min(nmx[w] + itole, ndat - 1);
    power_sums(X, Y, wei, imn, imx, low[w], nd, xs, xys, swei);
    xs[0] = 1.0;
    const int nu = w + 1;
    const double dx = high[w] - low[w];
    const int m = nd + 3;
    std::vector<double> A((size_t)m * m, 0.0), B(m, 0.0);
    auto Am = [&](int a, int b) -> double& { return A[(size_t)a * m + b]; };
    for (int a = 0; a <= nd; ++a)
      for (int b = 0; b <= nd; ++b) Am(a, b) = xs[a + b];
    for (int a = 0; a <= nd; ++a) Am(a, nd + 1) = -ipow(dx, a) * swei * 0.5;
    Am(0, nd + 2) = 0.0;
    for (int a = 1; a <= nd; ++a) Am(a, nd + 2) = -(a * ipow(dx, a - 1)) * swei * 0.5;
    for (int a = 0; a <= nd; ++a) Am(nd + 1, a) = ipow(dx, a);
    Am(nd + 2, 0) = 0.0;
    for (int a = 1; a <= nd; ++a) Am(nd + 2, a) = a * ipow(dx, a - 1);
    for (int a = 0; a <= nd; ++a) B[a] = xys[a];
    B[nd + 1] = C(0, nu);
    B[nd + 2] = C(1, nu);
    minver(A, m);
    for (int a = 0; a <= nd; ++a) {
      double s = 0.0;
      for (int b = 0; b < m; ++b) s += Am(a, b) * B[b];
      C(a, w) = s;
    }
  }
  // residual errors (:196-247): first window, last window, the ones between
  if (resid) {
    double r1 = 0.0, r2 = 0.0;
    auto acc = [&](int i, int w) {
      double ex = 0.0;
      const double dx = X[i] - low[w];
      for (int a = 0; a <= nd; ++a) ex += C(a, w) * ipow(dx, a);
      ex = Y[i] - ex;
      double ex2 = ex * ex;
      ex = ex2 * wei[i];
      ex2 = ex * ex2;
      r1 += ex;
      r2 += ex2;
    };
    for (int i = 0; i <= nmx[0]; ++i) acc(i, 0);
    if (nw > 1) {
      for (int i = nmx[nw - 2] + 1; i < ndat; ++i) acc(i, nw - 1);
      for (int w = 1; w < nw - 1; ++w)
        for (int i = nmx[w - 1] + 1; i <= nmx[w]; ++i) acc(i, w);
    }
    double sw = 0.0;
    for (int i = 0; i < ndat; ++i) sw += wei[i];
    r1 /= sw;
    r2 = std::sqrt(r2 / sw);
    resid[1] = std::sqrt(r2 - r1);
    resid[0] = std::sqrt(r1);
  }
  return JP_OK;
}

extern "C" int jp_ge_dlnn(const double *hist, const jp_ge_fit_params *fp, const jp_ge *old,
                          double *xo, double *yo, double *wo, int32_t *ndat) {
  if (!hist || !fp || !old || !xo || !yo || !wo || !ndat) return JP_E_INVALID;
  const int nbin = fp->nbin, nbor = fp->nbor;
  if (nbin < 2 || nbor < 0 || !(fp->emax > fp->emin) || !(fp->next_emax > fp->next_emin))
    return JP_E_INVALID;
  if (old->nwindow < 1 || old->ndeg < 0 || !old->coef || !old->low || !old->high ||
      !(old->ceup > old->celw))
    return JP_E_INVALID;
  const int nab = nbin + 2 * nbor;
  const double de = (fp->emax - fp->emin) / nbin;
  const double minec = fp->emin - de * nbor;
  std::vector<double> ee(nab), lnp(nab), dlnn(nab, 0.0);
  double pmax = 0.0;
  for (int i = 0; i < nab; ++i) {
    ee[i] = minec + de * (i + 0.5);
    pmax = std::max(pmax, hist[i]);
  }
  if (!(pmax > 0.0)) return JP_E_INVALID;
  const double lpmax = std::log(pmax);
  for (int i = 0; i < nab; ++i) lnp[i] = hist[i] == 0.0 ? 1.0 : std::log(hist[i]) - lpmax;
  // d lnN/dE of the weight the histogram was sampled with, at the upper edge of each bin
  const int onw = old->nwindow, ond = old->ndeg;
  int jw = 0;
  for (int i = 0; i < nab - 1; ++i) {
    const double xs = (ee[i] + 0.5 * de - old->celw) / (old->ceup - old->celw);
    double pold;
    if (xs < 0.0) {
      pold = old->alphalw;
    } else if (xs > 1.0) {
      pold = old->alphaup;
    } else {
      while (jw != onw - 1 && xs >= old->high[jw]) ++jw;
      const double dx = xs - old->low[jw];
      pold = old->coef[(size_t)jw * (ond + 1)];
      for (int k = 1; k <= ond; ++k) pold += old->coef[(size_t)jw * (ond + 1) + k] * ipow(dx, k);
    }
    if (lnp[i] != 1.0 && lnp[i + 1] != 1.0) dlnn[i] = (lnp[i + 1] - lnp[i]) / de + pold;
    else dlnn[i] = (xs >= 0.0 && xs <= 1.0) ? pold : 0.0;
  }
  // data on the next range
  const int ist = fp->neglect_low ? nbor : 0;
  const int ien = fp->neglect_high ? nbor + nbin - 1 : nab - 2;
  int n = 0;
  for (int i = ist; i <= ien; ++i) {
    const double x2 = (ee[i] + 0.5 * de - fp->next_emin) / (fp->next_emax - fp->next_emin);
    const double cnt = hist[i] + hist[i + 1];
    double wv;
    if (fp->ignore_empty) {
      if (dlnn[i] == 0.0) continue;
      wv = std::sqrt(cnt);
    } else {
      if (dlnn[i] == 0.0 && (x2 < old->celw || x2 > old->ceup)) continue;
      wv = std::max(std::sqrt(cnt), 1.0);
    }
    xo[n] = x2; yo[n] = dlnn[i]; wo[n] = wv;
    ++n;
  }
  *ndat = n;
  return JP_OK;
}

extern "C" int jp_ge_fit(const double *hist, const jp_ge_fit_params *fp, const jp_ge *old,
                         double *coef, double *low, double *high, jp_ge *out, double *resid) {
  if (!hist || !fp || !old || !coef || !low || !high || !out) return JP_E_INVALID;
  const int nw = fp->nwindow, nd = fp->ndeg;
  if (fp->nbin < 2 || fp->nbor < 0 || nw < 1 || nw > JP_GE_MAX_WINDOWS || nd < 1 ||
      nd > JP_GE_MAX_DEG)
    return JP_E_INVALID;
  const int cap = fp->nbin + 2 * fp->nbor;
  std::vector<double> X(cap), Y(cap), W(cap);
  int32_t ndat = 0;
  const int rd = jp_ge_dlnn(hist, fp, old, X.data(), Y.data(), W.data(), &ndat);
  if (rd) return rd;
  if (ndat < 2 * nw * (nd + 1)) return JP_E_INVALID;
  double r[2] = {0.0, 0.0};
  const int rc = jp_lstsq_windows(nw, ndat, nd, 0.0, 1.0, X.data(), Y.data(), W.data(), coef, low,
                                  high, r);
  if (rc) return rc;
  if (resid) { resid[0] = r[0]; resid[1] = r[1]; }
  double upd = coef[(size_t)(nw - 1) * (nd + 1)];
  const double dx = 1.0 - low[nw - 1];
  for (int k = 1; k <= nd; ++k) upd += coef[(size_t)(nw - 1) * (nd + 1) + k] * ipow(dx, k);
  out->nwindow = nw;
  out->ndeg = nd;
  out->coef = coef;
  out->low = low;
  out->high = high;
  out->alphalw = coef[0];
  out->alphaup = upd;
  out->celw = fp->next_emin;
  out->ceup = fp->next_emax;
  out->tempce = fp->next_temp;
  out->lower = old->lower;
  out->upper = old->upper;
  for (int i = 0; i < nw * (nd + 1); ++i)
    if (!std::isfinite(coef[i])) return JP_E_NONFINITE;
  return JP_OK;
}
