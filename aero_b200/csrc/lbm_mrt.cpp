// lbm_mrt.cpp -- MRT collision operator in the even/odd pair basis.
//
// The reference relaxes in moment space, f_post = Minv (m - S (m - m_eq)),
// m = M f (aero/lbm/kernels_mrt.py:190-241, kernels3d_mrt.py:24-82) with
//   D2Q9 : M9 of aero/lbm/mrt2d.py:36-46, Minv = inverse, S = build_s_vec
//   D3Q19: M19 of aero/lbm/mrt3d.py:46-87 (rank 16), Minv = Moore-Penrose
//          pseudo-inverse (mrt3d.py:91), S = build_s3_vec.
// That is f_post = A f + B feq with A = Minv (I - S) M, B = Minv S M.  Every
// moment row is either even or odd under e -> -e, so in the basis
//   s_0 = f_0,  s_p = f_i + f_opp(i),  t_p = f_i - f_opp(i)
// A and B are block diagonal (even 10x10 + odd 9x9 for D3Q19).  B acting on
// the equilibrium only needs its 7 even / 3 odd velocity moments, so the
// kernel evaluates s' = Ae s + Ce me, t' = Ao t + Co mo (278 FMA per D3Q19
// cell instead of two dense 19x19 products).  Because Minv M is a projector
// that keeps the rest state, the same operator applies to deviations f - w.
//
// The basis matrices are built here from the moment definitions, and the
// pseudo-inverse by a one-sided (Hestenes) Jacobi SVD, so the library needs
// no LAPACK.
#include <cmath>
#include <cstring>
#include <vector>

#include "lbm_lattice.cuh"
#include "lbm_params.h"

namespace aero {

namespace {

using Mat = std::vector<double>;  // row-major

template <class L>
void moment_basis(Mat &M) {
  const int Q = L::Q;
  M.assign(Q * Q, 0.0);
  for (int i = 0; i < Q; i++) {
    const int ex = L::ex[i], ey = L::ey[i], ez = L::ez[i];
    const int e2 = ex * ex + ey * ey + ez * ez;
    auto set = [&](int row, double v) { M[row * Q + i] = v; };
    if (L::DIMS == 2) {
      // rho, e, eps, jx, qx, jy, qy, pxx, pxy  (Lallemand & Luo ordering)
      set(0, 1);
      set(1, 3.0 * e2 - 4.0);
      set(2, (9.0 * e2 * e2 - 21.0 * e2 + 8.0) / 2.0);
      set(3, ex);
      set(4, (3.0 * e2 - 5.0) * ex);
      set(5, ey);
      set(6, (3.0 * e2 - 5.0) * ey);
      set(7, ex * ex - ey * ey);
      set(8, ex * ey);
    } else {
      // rho, e, eps, jx, qx, jy, qy, jz, qz, 3pxx, pww, pxy, pyz, pxz,
      // mx, my, mz, txxy, txyy  (row list of the reference basis)
      set(0, 1);
      set(1, 19.0 * e2 - 30.0);
      set(2, (21.0 * e2 * e2 - 53.0 * e2 + 24.0) / 2.0);
      set(3, ex);
      set(4, (5.0 * e2 - 9.0) * ex);
      set(5, ey);
      set(6, (5.0 * e2 - 9.0) * ey);
      set(7, ez);
      set(8, (5.0 * e2 - 9.0) * ez);
      set(9, 3.0 * ex * ex - e2);
      set(10, ey * ey - ez * ez);
      set(11, ex * ey);
      set(12, ey * ez);
      set(13, ex * ez);
      set(14, (3.0 * e2 - 5.0) * ex);
      set(15, (3.0 * e2 - 5.0) * ey);
      set(16, (3.0 * e2 - 5.0) * ez);
      set(17, ex * (ey * ey - ez * ez));
      set(18, ey * (ex * ex - ez * ez));
    }
  }
}

template <class L>
void relax_vector(double omega, std::vector<double> &s) {
  if (L::DIMS == 2) {
    const double sq = 8.0 * (2.0 - omega) / (8.0 - omega);
    s = {1.0, 1.64, 1.54, 1.0, sq, 1.0, sq, omega, omega};
  } else {
    s = {1.0, 1.19, 1.40, 1.0, 1.20, 1.0, 1.20, 1.0, 1.20, omega, omega,
         omega, omega, omega, 1.0, 1.0, 1.0, 1.0, 1.0};
  }
}

// Moore-Penrose pseudo-inverse of an n x n matrix by one-sided Jacobi SVD
// (Hestenes 1958): orthogonalise the columns of A V by plane rotations, then
// A = U Sigma V^T with the column norms as singular values.  Singular values
// below n * eps * sigma_max are treated as zero (the rank cut numpy uses).
void pinv(const Mat &A, int n, Mat &out) {
  Mat W = A;  // working columns
  Mat V(n * n, 0.0);
  for (int i = 0; i < n; i++) V[i * n + i] = 1.0;
  for (int sweep = 0; sweep < 60; sweep++) {
    double off = 0.0;
    for (int p = 0; p < n - 1; p++)
      for (int q = p + 1; q < n; q++) {
        double a = 0, b = 0, c = 0;
        for (int k = 0; k < n; k++) {
          a += W[k * n + p] * W[k * n + p];
          b += W[k * n + q] * W[k * n + q];
          c += W[k * n + p] * W[k * n + q];
        }
        if (std::fabs(c) <= 1e-300 || std::fabs(c) <= 1e-17 * std::sqrt(a * b)) continue;
        off = std::fmax(off, std::fabs(c) / std::sqrt(a * b));
        const double zeta = (b - a) / (2.0 * c);
        const double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
        const double cs = 1.0 / std::sqrt(1.0 + t * t), sn = cs * t;
        for (int k = 0; k < n; k++) {
          const double wp = W[k * n + p], wq = W[k * n + q];
          W[k * n + p] = cs * wp - sn * wq;
          W[k * n + q] = sn * wp + cs * wq;
          const double vp = V[k * n + p], vq = V[k * n + q];
          V[k * n + p] = cs * vp - sn * vq;
          V[k * n + q] = sn * vp + cs * vq;
        }
      }
    if (off < 1e-16) break;
  }
  std::vector<double> sig(n);
  double smax = 0.0;
  for (int j = 0; j < n; j++) {
    double a = 0;
    for (int k = 0; k < n; k++) a += W[k * n + j] * W[k * n + j];
    sig[j] = std::sqrt(a);
    smax = std::fmax(smax, sig[j]);
  }
  const double cut = n * 2.220446049250313e-16 * smax;
  out.assign(n * n, 0.0);
  // A = U S V^T, U_j = W_j / s_j  =>  A+ = sum_j V_j U_j^T / s_j = sum_j V_j W_j^T / s_j^2
  for (int j = 0; j < n; j++) {
    if (sig[j] <= cut) continue;
    const double inv2 = 1.0 / (sig[j] * sig[j]);
    for (int r = 0; r < n; r++)
      for (int c = 0; c < n; c++) out[r * n + c] += V[r * n + j] * W[c * n + j] * inv2;
  }
}

void matmul(const Mat &A, const Mat &B, int n, Mat &C) {
  C.assign(n * n, 0.0);
  for (int r = 0; r < n; r++)
    for (int k = 0; k < n; k++) {
      const double a = A[r * n + k];
      if (a == 0.0) continue;
      for (int c = 0; c < n; c++) C[r * n + c] += a * B[k * n + c];
    }
}

template <class L>
bool build(double omega, MrtCoeffs<double> &out, double *A_full, double *B_full) {
  const int Q = L::Q, NE = L::NP + 1, NO = L::NP;
  const int KE = L::DIMS == 2 ? 4 : 7, KO = L::DIMS;
  Mat M, Minv;
  moment_basis<L>(M);
  std::vector<double> s;
  relax_vector<L>(omega, s);
  pinv(M, Q, Minv);
  Mat ImS(Q * Q, 0.0), SM(Q * Q, 0.0);
  for (int r = 0; r < Q; r++)
    for (int c = 0; c < Q; c++) {
      ImS[r * Q + c] = (1.0 - s[r]) * M[r * Q + c];
      SM[r * Q + c] = s[r] * M[r * Q + c];
    }
  Mat A, B;
  matmul(Minv, ImS, Q, A);
  matmul(Minv, SM, Q, B);
  if (A_full) std::memcpy(A_full, A.data(), sizeof(double) * Q * Q);
  if (B_full) std::memcpy(B_full, B.data(), sizeof(double) * Q * Q);
  // pair basis: row k of U gives s_k (k < NE) or t_{k-NE}
  Mat U(Q * Q, 0.0), Uinv(Q * Q, 0.0);
  U[0] = 1.0;
  Uinv[0] = 1.0;
  for (int k = 0; k < NO; k++) {
    const int i = L::pair[k], o = L::opp[L::pair[k]];
    U[(k + 1) * Q + i] = 1.0;
    U[(k + 1) * Q + o] = 1.0;
    U[(NE + k) * Q + i] = 1.0;
    U[(NE + k) * Q + o] = -1.0;
    // f_i = (s + t) / 2, f_o = (s - t) / 2
    Uinv[i * Q + (k + 1)] = 0.5;
    Uinv[i * Q + (NE + k)] = 0.5;
    Uinv[o * Q + (k + 1)] = 0.5;
    Uinv[o * Q + (NE + k)] = -0.5;
  }
  Mat T, Ap, Bp;
  matmul(U, A, Q, T);
  matmul(T, Uinv, Q, Ap);
  matmul(U, B, Q, T);
  matmul(T, Uinv, Q, Bp);
  double offmax = 0.0;
  for (int r = 0; r < Q; r++)
    for (int c = 0; c < Q; c++)
      if ((r < NE) != (c < NE)) offmax = std::fmax(offmax, std::fmax(std::fabs(Ap[r * Q + c]), std::fabs(Bp[r * Q + c])));
  if (offmax > 1e-12) return false;
  // equilibrium moments: seq = G me, teq = H mo (deviation form, rest weights cancel)
  std::vector<double> G(NE * KE, 0.0), H(NO * KO, 0.0);
  for (int k = 0; k < NE; k++) {
    const int i = k == 0 ? 0 : L::pair[k - 1];
    const double ww = k == 0 ? L::w[0] : 2.0 * L::w[i];
    const double ex = L::ex[i], ey = L::ey[i], ez = L::ez[i];
    G[k * KE + 0] = ww;
    G[k * KE + 1] = ww * (4.5 * ex * ex - 1.5);
    G[k * KE + 2] = ww * (4.5 * ey * ey - 1.5);
    if (L::DIMS == 2) {
      G[k * KE + 3] = ww * 9.0 * ex * ey;
    } else {
      G[k * KE + 3] = ww * (4.5 * ez * ez - 1.5);
      G[k * KE + 4] = ww * 9.0 * ex * ey;
      G[k * KE + 5] = ww * 9.0 * ex * ez;
      G[k * KE + 6] = ww * 9.0 * ey * ez;
    }
  }
  for (int k = 0; k < NO; k++) {
    const int i = L::pair[k];
    H[k * KO + 0] = 6.0 * L::w[i] * L::ex[i];
    H[k * KO + 1] = 6.0 * L::w[i] * L::ey[i];
    if (L::DIMS == 3) H[k * KO + 2] = 6.0 * L::w[i] * L::ez[i];
  }
  std::memset(&out, 0, sizeof(out));
  for (int r = 0; r < NE; r++) {
    for (int c = 0; c < NE; c++) out.Ae[r * 10 + c] = Ap[r * Q + c];
    for (int k = 0; k < KE; k++) {
      double a = 0;
      for (int c = 0; c < NE; c++) a += Bp[r * Q + c] * G[c * KE + k];
      out.Ce[r * 7 + k] = a;
    }
  }
  for (int r = 0; r < NO; r++) {
    for (int c = 0; c < NO; c++) out.Ao[r * 9 + c] = Ap[(NE + r) * Q + NE + c];
    for (int k = 0; k < KO; k++) {
      double a = 0;
      for (int c = 0; c < NO; c++) a += Bp[(NE + r) * Q + NE + c] * H[c * KO + k];
      out.Co[r * 3 + k] = a;
    }
  }
  return true;
}

// D3Q19 blocks in the cubic-symmetry-adapted basis.  From the pair-basis
// blocks (even Ae/Be 10x10 on s, odd Ao/Bo 9x9 on t) the change of basis
//   g = V s: rest, face sum, edge sum, face doublet (2X-Y-Z, Y-Z), edge
//            doublet (2Pyz-Pxz-Pxy, Pxz-Pxy), shear differences (3)
//   h = W t: face differences (3), momentum-like edge sums (3), remaining
//            odd edge combinations (3)
// makes the operator block diagonal.  Every entry outside the expected
// blocks, every mismatch between blocks that symmetry makes equal, and any
// non-zero on the last three odd coordinates is rejected.
bool build_adapted(const Mat &Ap, const Mat &Bp, Mrt3Adapted<double> &m) {
  const int Q = 19;
  double V[10][10] = {{0}}, W[9][9] = {{0}};
  V[0][0] = 1;
  V[1][1] = V[1][2] = V[1][3] = 1;
  for (int k = 4; k < 10; k++) V[2][k] = 1;
  V[3][1] = 2; V[3][2] = -1; V[3][3] = -1;
  V[4][2] = 1; V[4][3] = -1;
  V[5][4] = V[5][5] = -1; V[5][6] = V[5][7] = -1; V[5][8] = V[5][9] = 2;
  V[6][4] = V[6][5] = -1; V[6][6] = V[6][7] = 1;
  V[7][4] = 1; V[7][5] = -1;
  V[8][6] = 1; V[8][7] = -1;
  V[9][8] = 1; V[9][9] = -1;
  // odd: t index k -> pair k (t4..t9 at columns 3..8)
  W[0][0] = 1; W[1][1] = 1; W[2][2] = 1;
  const double xy_x[9] = {0, 0, 0, 1, -1, 0, 0, 0, 0}, xz_x[9] = {0, 0, 0, 0, 0, 1, -1, 0, 0};
  const double xy_y[9] = {0, 0, 0, 1, 1, 0, 0, 0, 0}, yz_y[9] = {0, 0, 0, 0, 0, 0, 0, 1, -1};
  const double xz_z[9] = {0, 0, 0, 0, 0, 1, 1, 0, 0}, yz_z[9] = {0, 0, 0, 0, 0, 0, 0, 1, 1};
  for (int k = 0; k < 9; k++) {
    W[3][k] = xy_x[k] + xz_x[k];
    W[4][k] = xy_y[k] + yz_y[k];
    W[5][k] = xz_z[k] + yz_z[k];
    W[6][k] = xy_x[k] - xz_x[k];
    W[7][k] = xy_y[k] - yz_y[k];
    W[8][k] = xz_z[k] - yz_z[k];
  }
  Mat Vm(100), Wm(81), Vi, Wi;
  for (int r = 0; r < 10; r++)
    for (int c = 0; c < 10; c++) Vm[r * 10 + c] = V[r][c];
  for (int r = 0; r < 9; r++)
    for (int c = 0; c < 9; c++) Wm[r * 9 + c] = W[r][c];
  pinv(Vm, 10, Vi);
  pinv(Wm, 9, Wi);
  Mat Ae(100), Be(100), Ao(81), Bo(81);
  for (int r = 0; r < 10; r++)
    for (int c = 0; c < 10; c++) {
      Ae[r * 10 + c] = Ap[r * Q + c];
      Be[r * 10 + c] = Bp[r * Q + c];
    }
  for (int r = 0; r < 9; r++)
    for (int c = 0; c < 9; c++) {
      Ao[r * 9 + c] = Ap[(10 + r) * Q + 10 + c];
      Bo[r * 9 + c] = Bp[(10 + r) * Q + 10 + c];
    }
  Mat T1, Aa, Ba, Oa, Ob;
  matmul(Vm, Ae, 10, T1); matmul(T1, Vi, 10, Aa);
  matmul(Vm, Be, 10, T1); matmul(T1, Vi, 10, Ba);
  matmul(Wm, Ao, 9, T1); matmul(T1, Wi, 9, Oa);
  matmul(Wm, Bo, 9, T1); matmul(T1, Wi, 9, Ob);
  // equilibrium: even pair-basis seq = G me_std, me_std = (drho, kxx, kyy, kzz, kxy, kxz, kyz)
  // with k_ab = rho u_a u_b; adapted inputs m_ad = (drho, ru2, mE1, mE2, kxy, kxz, kyz)
  double G[10][7] = {{0}};
  for (int k = 0; k < 10; k++) {
    const int i = k == 0 ? 0 : D3Q19::pair[k - 1];
    const double ww = k == 0 ? D3Q19::w[0] : 2.0 * D3Q19::w[i];
    const double ex = D3Q19::ex[i], ey = D3Q19::ey[i], ez = D3Q19::ez[i];
    G[k][0] = ww;
    G[k][1] = ww * (4.5 * ex * ex - 1.5);
    G[k][2] = ww * (4.5 * ey * ey - 1.5);
    G[k][3] = ww * (4.5 * ez * ez - 1.5);
    G[k][4] = ww * 9.0 * ex * ey;
    G[k][5] = ww * 9.0 * ex * ez;
    G[k][6] = ww * 9.0 * ey * ez;
  }
  const double Tm[7][7] = {{1, 0, 0, 0, 0, 0, 0},
                           {0, 1.0 / 3, 1.0 / 3, 0, 0, 0, 0},
                           {0, 1.0 / 3, -1.0 / 6, 0.5, 0, 0, 0},
                           {0, 1.0 / 3, -1.0 / 6, -0.5, 0, 0, 0},
                           {0, 0, 0, 0, 1, 0, 0},
                           {0, 0, 0, 0, 0, 1, 0},
                           {0, 0, 0, 0, 0, 0, 1}};
  double K[10][7] = {{0}};  // adapted outputs x adapted inputs
  for (int r = 0; r < 10; r++)
    for (int q = 0; q < 7; q++) {
      double acc = 0;
      for (int a = 0; a < 10; a++) {
        double vb = 0;  // (Ba V)[r][a]
        for (int b = 0; b < 10; b++) vb += Ba[r * 10 + b] * Vm[b * 10 + a];
        double gt = 0;  // (G Tm)[a][q]
        for (int c = 0; c < 7; c++) gt += G[a][c] * Tm[c][q];
        acc += vb * gt;
      }
      K[r][q] = acc;
    }
  // odd equilibrium: teq = H (rho u), H[k][a] = 6 w e_a of pair k
  double Ko[9][3] = {{0}};
  for (int r = 0; r < 9; r++)
    for (int q = 0; q < 3; q++) {
      double acc = 0;
      for (int a = 0; a < 9; a++) {
        double wb = 0;
        for (int b = 0; b < 9; b++) wb += Ob[r * 9 + b] * Wm[b * 9 + a];
        const int i = D3Q19::pair[a];
        const double e = q == 0 ? D3Q19::ex[i] : (q == 1 ? D3Q19::ey[i] : D3Q19::ez[i]);
        acc += wb * 6.0 * D3Q19::w[i] * e;
      }
      Ko[r][q] = acc;
    }
  // --- expected structure -------------------------------------------------
  auto eb = [](int r) { return r < 3 ? 0 : (r == 3 || r == 5) ? 1 : (r == 4 || r == 6) ? 2 : r; };
  auto ob = [](int r) { return r == 0 || r == 3 ? 0 : (r == 1 || r == 4) ? 1 : (r == 2 || r == 5) ? 2 : r; };
  double scale = 0, err = 0;
  for (int r = 0; r < 10; r++)
    for (int c = 0; c < 10; c++) {
      scale = std::fmax(scale, std::fabs(Aa[r * 10 + c]));
      if (eb(r) != eb(c)) err = std::fmax(err, std::fabs(Aa[r * 10 + c]));
    }
  for (int r = 0; r < 9; r++)
    for (int c = 0; c < 9; c++)
      if (ob(r) != ob(c) || r >= 6) err = std::fmax(err, std::fabs(Oa[r * 9 + c]));
  auto A = [&](int r, int c) { return Aa[r * 10 + c]; };
  auto O = [&](int r, int c) { return Oa[r * 9 + c]; };
  // doublet components share one block; triplets share one block
  err = std::fmax(err, std::fabs(A(3, 3) - A(4, 4)));
  err = std::fmax(err, std::fabs(A(3, 5) - A(4, 6)));
  err = std::fmax(err, std::fabs(A(5, 3) - A(6, 4)));
  err = std::fmax(err, std::fabs(A(5, 5) - A(6, 6)));
  err = std::fmax(err, std::fmax(std::fabs(A(7, 7) - A(8, 8)), std::fabs(A(7, 7) - A(9, 9))));
  for (int q = 1; q < 3; q++) {
    err = std::fmax(err, std::fabs(O(0, 0) - O(q, q)));
    err = std::fmax(err, std::fabs(O(0, 3) - O(q, 3 + q)));
    err = std::fmax(err, std::fabs(O(3, 0) - O(3 + q, q)));
    err = std::fmax(err, std::fabs(O(3, 3) - O(3 + q, 3 + q)));
  }
  // equilibrium couplings: A1 rows take (drho, ru2); doublets take mE1 / mE2
  // with equal weights; shear rows take their own k; nothing else
  for (int r = 0; r < 10; r++)
    for (int q = 0; q < 7; q++) {
      const bool allowed = (r < 3 && q < 2) || ((r == 3 || r == 5) && q == 2) || ((r == 4 || r == 6) && q == 3) ||
                           (r >= 7 && q == r - 3);
      if (!allowed) err = std::fmax(err, std::fabs(K[r][q]));
    }
  err = std::fmax(err, std::fabs(K[3][2] - K[4][3]));
  err = std::fmax(err, std::fabs(K[5][2] - K[6][3]));
  err = std::fmax(err, std::fmax(std::fabs(K[7][4] - K[8][5]), std::fabs(K[7][4] - K[9][6])));
  for (int r = 0; r < 9; r++)
    for (int q = 0; q < 3; q++) {
      const bool allowed = (r < 3 && q == r) || (r >= 3 && r < 6 && q == r - 3);
      if (!allowed) err = std::fmax(err, std::fabs(Ko[r][q]));
    }
  for (int q = 1; q < 3; q++) {
    err = std::fmax(err, std::fabs(Ko[0][0] - Ko[q][q]));
    err = std::fmax(err, std::fabs(Ko[3][0] - Ko[3 + q][q]));
  }
  if (!(err <= 1e-12 * std::fmax(scale, 1.0))) return false;
  for (int r = 0; r < 3; r++) {
    for (int c = 0; c < 3; c++) m.a1[r * 3 + c] = A(r, c);
    m.ca1[r * 2 + 0] = K[r][0];
    m.ca1[r * 2 + 1] = K[r][1];
  }
  m.e[0] = A(3, 3); m.e[1] = A(3, 5); m.e[2] = A(5, 3); m.e[3] = A(5, 5);
  m.ce[0] = K[3][2]; m.ce[1] = K[5][2];
  m.t2 = A(7, 7); m.ct2 = K[7][4];
  m.v[0] = O(0, 0); m.v[1] = O(0, 3); m.v[2] = O(3, 0); m.v[3] = O(3, 3);
  m.cv[0] = Ko[0][0]; m.cv[1] = Ko[3][0];
  return true;
}

}  // namespace

bool build_mrt3_adapted(double omega, Mrt3Adapted<double> &m) {
  // pair-basis operator of the reference D3Q19 basis
  const int Q = 19;
  Mat M, Minv;
  moment_basis<D3Q19>(M);
  std::vector<double> s;
  relax_vector<D3Q19>(omega, s);
  pinv(M, Q, Minv);
  Mat ImS(Q * Q), SM(Q * Q);
  for (int r = 0; r < Q; r++)
    for (int c = 0; c < Q; c++) {
      ImS[r * Q + c] = (1.0 - s[r]) * M[r * Q + c];
      SM[r * Q + c] = s[r] * M[r * Q + c];
    }
  Mat A, B, U(Q * Q, 0.0), Uinv(Q * Q, 0.0), T, Ap, Bp;
  matmul(Minv, ImS, Q, A);
  matmul(Minv, SM, Q, B);
  const int NE = 10;
  U[0] = 1.0;
  Uinv[0] = 1.0;
  for (int k = 0; k < 9; k++) {
    const int i = D3Q19::pair[k], o = D3Q19::opp[i];
    U[(k + 1) * Q + i] = 1.0;
    U[(k + 1) * Q + o] = 1.0;
    U[(NE + k) * Q + i] = 1.0;
    U[(NE + k) * Q + o] = -1.0;
    Uinv[i * Q + (k + 1)] = 0.5;
    Uinv[i * Q + (NE + k)] = 0.5;
    Uinv[o * Q + (k + 1)] = 0.5;
    Uinv[o * Q + (NE + k)] = -0.5;
  }
  matmul(U, A, Q, T);
  matmul(T, Uinv, Q, Ap);
  matmul(U, B, Q, T);
  matmul(T, Uinv, Q, Bp);
  return build_adapted(Ap, Bp, m);
}

bool build_mrt(int dims, double omega, MrtCoeffs<double> &out, double *A_full, double *B_full) {
  return dims == 2 ? build<D2Q9>(omega, out, A_full, B_full) : build<D3Q19>(omega, out, A_full, B_full);
}

bool mrt_pinv_basis(int dims, double *M_out, double *Minv_out) {
  Mat M, Minv;
  int Q;
  if (dims == 2) {
    moment_basis<D2Q9>(M);
    Q = 9;
  } else {
    moment_basis<D3Q19>(M);
    Q = 19;
  }
  pinv(M, Q, Minv);
  std::memcpy(M_out, M.data(), sizeof(double) * Q * Q);
  std::memcpy(Minv_out, Minv.data(), sizeof(double) * Q * Q);
  return true;
}

}  // namespace aero
