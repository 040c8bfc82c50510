// Eigenvalues of a complex Hermitian band matrix in a window (vl, vu]: the
// host-side solve of the block Lanczos band (block-tridiagonal) matrix,
// which the reference hands to LAPACK zhbevx with RANGE='V', UPLO='L'
// (solve_block_tridiagonal_eigenvalues, NEMO_3D/eigen/src/lanczos_blk.c:
// 891-991).  Written from the method, not from LAPACK: the band is reduced
// to Hermitian tridiagonal form by Givens rotations that chase each bulge
// down the band (Schwarz's band reduction), the tridiagonal is made real by
// a diagonal unitary similarity (|e_i|), and the eigenvalues in the window
// are found by Sturm-count bisection.  O(n^2 kd) work, O(n kd) memory.
#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

#include "tbgpu_internal.cuh"

namespace tbgpu {

using cplx = std::complex<double>;

namespace {

// Lower band storage with room for one bulge diagonal: element (i, j),
// j <= i <= j + w, at a[j * (w + 1) + (i - j)], w = kd + 1.
struct Band {
  int n, w;
  std::vector<cplx> a;
  Band(int n_, int kd) : n(n_), w(kd + 1), a(size_t(n_) * (kd + 2), cplx(0.0, 0.0)) {}
  bool in(int i, int j) const { return i >= j ? i - j <= w : j - i <= w; }
  cplx get(int i, int j) const {
    if (i >= j) return i - j <= w ? a[size_t(j) * (w + 1) + (i - j)] : cplx(0.0, 0.0);
    return j - i <= w ? std::conj(a[size_t(i) * (w + 1) + (j - i)]) : cplx(0.0, 0.0);
  }
  void set(int i, int j, cplx v) {
    if (i >= j)
      a[size_t(j) * (w + 1) + (i - j)] = v;
    else
      a[size_t(i) * (w + 1) + (j - i)] = std::conj(v);
  }
};

// Rotation G on rows/columns (p, p+1) with G = [c, s; -conj(s), c] chosen so
// that (G x)[1] = 0 for x = (x0, x1); returns false when x1 is already 0.
bool givens(cplx x0, cplx x1, double &c, cplx &s) {
  const double a0 = std::abs(x0), a1 = std::abs(x1);
  if (a1 == 0.0) return false;
  const double r = std::hypot(a0, a1);
  if (a0 == 0.0) {
    c = 0.0;
    s = std::conj(x1) / a1;  // maps (0, x1) to (|x1|, 0)
    return true;
  }
  c = a0 / r;
  s = (x0 / a0) * std::conj(x1) / r;
  return true;
}

// A <- G A G^H on rows/columns p, q = p + 1, for the band entries that can
// be nonzero (columns within w of p or q).
void rotate(Band &B, int p, double c, cplx s) {
  const int q = p + 1, n = B.n, w = B.w;
  const int lo = std::max(0, p - w), hi = std::min(n - 1, q + w);
  for (int m = lo; m <= hi; m++) {
    if (m == p || m == q) continue;
    const bool ip = B.in(p, m), iq = B.in(q, m);
    if (!ip && !iq) continue;
    const cplx ap = B.get(p, m), aq = B.get(q, m);
    // row update: [ap'; aq'] = G [ap; aq]
    const cplx np = c * ap + s * aq;
    const cplx nq = -std::conj(s) * ap + c * aq;
    if (ip) B.set(p, m, np);
    if (iq) B.set(q, m, nq);
  }
  const cplx app = B.get(p, p), aqq = B.get(q, q), aqp = B.get(q, p), apq = std::conj(aqp);
  // 2x2 block: G [app apq; aqp aqq] G^H
  const cplx t00 = c * app + s * aqp, t01 = c * apq + s * aqq;
  const cplx t10 = -std::conj(s) * app + c * aqp, t11 = -std::conj(s) * apq + c * aqq;
  const cplx n00 = t00 * c + t01 * std::conj(s);
  const cplx n10 = t10 * c + t11 * std::conj(s);
  const cplx n11 = -t10 * s + t11 * c;
  B.set(p, p, cplx(n00.real(), 0.0));
  B.set(q, q, cplx(n11.real(), 0.0));
  B.set(q, p, n10);
}

int sturm_count(const std::vector<double> &d, const std::vector<double> &e2, double x) {
  const int n = int(d.size());
  int cnt = 0;
  double q = d[0] - x;
  if (q < 0) cnt++;
  for (int i = 1; i < n; i++) {
    if (std::fabs(q) < 1e-300) q = q < 0 ? -1e-300 : 1e-300;
    q = d[i] - x - e2[i - 1] / q;
    if (q < 0) cnt++;
  }
  return cnt;
}

}  // namespace

int band_eigenvalues(int n, int kd, const cplx *ab, double vl, double vu, double abstol,
                     std::vector<double> &w) {
  w.clear();
  if (n <= 0 || kd < 0) return TBGPU_E_ARG;
  Band B(n, kd);
  for (int j = 0; j < n; j++)
    for (int i = j; i <= std::min(n - 1, j + kd); i++) B.set(i, j, ab[size_t(j) * (kd + 1) + (i - j)]);
  for (int j = 0; j < n; j++) B.set(j, j, cplx(B.get(j, j).real(), 0.0));
  // reduce: clear column j below the first subdiagonal, chasing the bulge
  for (int j = 0; j + 2 < n; j++) {
    for (int k = std::min(kd, n - 1 - j); k >= 2; k--) {
      int row = j + k, col = j;
      // annihilate (row, col) with a rotation of rows row-1, row; the fill
      // it creates at (row + kd, row - 1) is chased down by kd each step
      while (row < n) {
        double c;
        cplx s;
        if (!givens(B.get(row - 1, col), B.get(row, col), c, s)) break;
        rotate(B, row - 1, c, s);
        B.set(row, col, cplx(0.0, 0.0));
        const int nrow = row + kd, ncol = row - 1;
        if (nrow >= n) break;
        row = nrow;
        col = ncol;
      }
    }
  }
  std::vector<double> d(n), e2(n > 1 ? n - 1 : 0);
  double gl = 1e300, gu = -1e300;
  for (int i = 0; i < n; i++) d[i] = B.get(i, i).real();
  for (int i = 0; i + 1 < n; i++) e2[i] = std::norm(B.get(i + 1, i));
  for (int i = 0; i < n; i++) {
    const double r = (i > 0 ? std::sqrt(e2[i - 1]) : 0.0) + (i + 1 < n ? std::sqrt(e2[i]) : 0.0);
    gl = std::min(gl, d[i] - r);
    gu = std::max(gu, d[i] + r);
  }
  const double lo = std::max(vl, gl - 1e-12), hi = std::min(vu, gu + 1e-12);
  if (!(hi > lo)) return TBGPU_OK;
  const int nlo = sturm_count(d, e2, lo), nhi = sturm_count(d, e2, hi);
  const double tol = std::max(abstol, 4e-16 * std::max(std::fabs(gl), std::fabs(gu)));
  for (int k = nlo; k < nhi; k++) {  // the k-th eigenvalue (0-based) lies in (lo, hi]
    double a = lo, b = hi;
    while (b - a > tol) {
      const double mid = 0.5 * (a + b);
      if (sturm_count(d, e2, mid) > k) b = mid; else a = mid;
    }
    w.push_back(0.5 * (a + b));
  }
  return TBGPU_OK;
}

}  // namespace tbgpu

extern "C" int tbgpu_band_eigenvalues(int n, int kd, const double *ab, double vl, double vu,
                                      double abstol, double *w, int cap) {
  using namespace tbgpu;
  if (!ab || !w || n <= 0 || kd < 0 || cap < 0) return set_error(TBGPU_E_ARG);
  std::vector<double> out;
  int rc = band_eigenvalues(n, kd, reinterpret_cast<const cplx *>(ab), vl, vu, abstol, out);
  if (rc) return set_error(rc);
  const int m = int(out.size());
  for (int i = 0; i < std::min(m, cap); i++) w[i] = out[i];
  return m;
}
