// Small dense complex inverse of the one-particle Green's functions.
#pragma once
#include "common.cuh"

#define GINV_MAXND 8

// ---------------------------------------------------------------------------
// G(k, nu) = (i nu + mu - H(k) - dc - Sigma(nu))^-1.  For ndim <= 3 the same
// closed cofactor forms as inverse_matrix_2/3 (src/aux.f90:288-325), else a
// Gauss-Jordan inverse with partial pivoting.
// ---------------------------------------------------------------------------
__device__ inline void ginv_small(int nd, z64 *a /* nd x nd col-major, in/out */) {
  if (nd == 1) {
    a[0] = crcp(a[0]);
  } else if (nd == 2) {
    z64 a11 = a[0], a21 = a[1], a12 = a[2], a22 = a[3];
    z64 det = csub(cmul(a11, a22), cmul(a12, a21));
    z64 di = crcp(det);
    a[0] = cmul(di, a22);
    a[1] = cneg(cmul(di, a21));
    a[2] = cneg(cmul(di, a12));
    a[3] = cmul(di, a11);
  } else if (nd == 3) {
#define A(i, j) a[(i - 1) + (j - 1) * 3]
    z64 det = cmul(cmul(A(1, 1), A(2, 2)), A(3, 3));
    det = csub(det, cmul(cmul(A(1, 1), A(2, 3)), A(3, 2)));
    det = csub(det, cmul(cmul(A(1, 2), A(2, 1)), A(3, 3)));
    det = cadd(det, cmul(cmul(A(1, 2), A(2, 3)), A(3, 1)));
    det = cadd(det, cmul(cmul(A(1, 3), A(2, 1)), A(3, 2)));
    det = csub(det, cmul(cmul(A(1, 3), A(2, 2)), A(3, 1)));
    z64 di = crcp(det);
    z64 b[9];
#define B(i, j) b[(i - 1) + (j - 1) * 3]
    B(1, 1) = cmul(di, csub(cmul(A(2, 2), A(3, 3)), cmul(A(2, 3), A(3, 2))));
    B(2, 1) = cneg(cmul(di, csub(cmul(A(2, 1), A(3, 3)), cmul(A(2, 3), A(3, 1)))));
    B(3, 1) = cmul(di, csub(cmul(A(2, 1), A(3, 2)), cmul(A(2, 2), A(3, 1))));
    B(1, 2) = cneg(cmul(di, csub(cmul(A(1, 2), A(3, 3)), cmul(A(1, 3), A(3, 2)))));
    B(2, 2) = cmul(di, csub(cmul(A(1, 1), A(3, 3)), cmul(A(1, 3), A(3, 1))));
    B(3, 2) = cneg(cmul(di, csub(cmul(A(1, 1), A(3, 2)), cmul(A(1, 2), A(3, 1)))));
    B(1, 3) = cmul(di, csub(cmul(A(1, 2), A(2, 3)), cmul(A(1, 3), A(2, 2))));
    B(2, 3) = cneg(cmul(di, csub(cmul(A(1, 1), A(2, 3)), cmul(A(1, 3), A(2, 1)))));
    B(3, 3) = cmul(di, csub(cmul(A(1, 1), A(2, 2)), cmul(A(1, 2), A(2, 1))));
#undef A
#undef B
    for (int i = 0; i < 9; ++i) a[i] = b[i];
  } else {
    // Gauss-Jordan with partial pivoting on [a | I]
    z64 inv[GINV_MAXND * GINV_MAXND];
    int n = nd;
    for (int i = 0; i < n * n; ++i) inv[i] = czero<z64>();
    for (int i = 0; i < n; ++i) inv[i + i * n] = make_double2(1.0, 0.0);
    for (int c = 0; c < n; ++c) {
      int p = c;
      double best = cabs1(a[c + c * n]);
      for (int r = c + 1; r < n; ++r) {
        double v = cabs1(a[r + c * n]);
        if (v > best) { best = v; p = r; }
      }
      if (p != c)
        for (int j = 0; j < n; ++j) {
          z64 t = a[c + j * n]; a[c + j * n] = a[p + j * n]; a[p + j * n] = t;
          t = inv[c + j * n]; inv[c + j * n] = inv[p + j * n]; inv[p + j * n] = t;
        }
      z64 r = crcp(a[c + c * n]);
      for (int j = 0; j < n; ++j) {
        a[c + j * n] = cmul(a[c + j * n], r);
        inv[c + j * n] = cmul(inv[c + j * n], r);
      }
      for (int rr = 0; rr < n; ++rr) {
        if (rr == c) continue;
        z64 f = a[rr + c * n];
        for (int j = 0; j < n; ++j) {
          cfms(a[rr + j * n], f, a[c + j * n]);
          cfms(inv[rr + j * n], f, inv[c + j * n]);
        }
      }
    }
    for (int i = 0; i < n * n; ++i) a[i] = inv[i];
  }
}

