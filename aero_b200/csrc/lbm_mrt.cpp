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

}  // namespace

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
