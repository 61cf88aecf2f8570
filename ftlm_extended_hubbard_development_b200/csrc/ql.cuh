// Implicit QL with shifts on a symmetric tridiagonal matrix, tracking only
// the first row of the eigenvector matrix (Golub-Welsch: the FTLM weights are
// the squared first components), then an ascending insertion sort. One
// thread per matrix. Shared by the engine's batched Ritz stage (lanczos.cu)
// and the allocation-free entry point (noalloc.cu).
#pragma once

namespace ftlm {

// d[0..n): diagonal, e[0..n-1): off-diagonal (e[n-1] = 0), z: first row of
// the eigenvector matrix (1, 0, ..., 0 on entry). A is any indexable view of
// doubles. Returns false when an eigenvalue needed more than 200 iterations.
template <typename A>
__device__ __forceinline__ bool ql_first_row(int n, A d, A z, A e) {
  bool ok = true;
  const double eps = 2.220446049250313e-16;
  for (int l = 0; l < n; ++l) {
    int iter = 0;
    while (true) {
      int m = l;
      for (; m < n - 1; ++m) {
        const double dd = fabs(d[m]) + fabs(d[m + 1]);
        if (fabs(e[m]) <= eps * dd) break;
      }
      if (m == l) break;
      if (++iter > 200) {
        ok = false;
        break;
      }
      double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
      double rr = hypot(g, 1.0);
      g = d[m] - d[l] + e[l] / (g + copysign(rr, g));
      double s = 1.0, c = 1.0, p = 0.0;
      bool underflow = false;
      for (int i = m - 1; i >= l; --i) {
        double f = s * e[i];
        const double b = c * e[i];
        rr = hypot(f, g);
        e[i + 1] = rr;
        if (rr == 0.0) {
          d[i + 1] -= p;
          e[m] = 0.0;
          underflow = true;
          break;
        }
        s = f / rr;
        c = g / rr;
        g = d[i + 1] - p;
        rr = (d[i] - g) * s + 2.0 * c * b;
        p = s * rr;
        d[i + 1] = g + p;
        g = c * rr - b;
        f = z[i + 1];
        z[i + 1] = s * z[i] + c * f;
        z[i] = c * z[i] - s * f;
      }
      if (underflow) continue;
      d[l] -= p;
      e[l] = g;
      e[m] = 0.0;
    }
  }
  for (int i = 1; i < n; ++i) {  // insertion sort, ascending
    const double dk = d[i], zk = z[i];
    int j = i - 1;
    while (j >= 0 && d[j] > dk) {
      d[j + 1] = d[j];
      z[j + 1] = z[j];
      --j;
    }
    d[j + 1] = dk;
    z[j + 1] = zk;
  }
  return ok;
}

}  // namespace ftlm
