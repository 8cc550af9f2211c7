// grid.cpp -- FP64 host math of the search: rotation matrices and the Euler search grid.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../../include/emc_b200.h"

namespace emc {
void set_error(const char* fmt, ...);

// MATLAB colon a:d:b (d > 0); empty when b < a.
static std::vector<double> colon(double a, double d, double b) {
  std::vector<double> v;
  if (!(d > 0) || b < a) return v;
  const double span = (b - a) / d;
  const long n = (long)floor(span + 1e-10 * (1.0 + fabs(span))) + 1;
  for (long k = 0; k < n; ++k) v.push_back(a + k * d);
  return v;
}
}  // namespace emc

extern "C" {

// BH_defineMatrix(ANGLES, 'Bah', DIRECTION) (coordinates/BH_defineMatrix.m:85-126).
emc_status emc_define_matrix(const double angles_deg[3], int direction, double R[9]) {
  if (!angles_deg || !R || (direction != 0 && direction != 1)) {
    emc::set_error("emc_define_matrix: bad argument");
    return EMC_E_ARG;
  }
  double a[3];
  for (int i = 0; i < 3; ++i) a[i] = angles_deg[i] * (M_PI / 180.0);
  if (direction == 0) {
    for (int i = 0; i < 3; ++i) a[i] = -a[i];
  } else {
    const double t = a[0];
    a[0] = a[2];
    a[2] = t;
  }
  const double c1 = cos(a[0]), s1 = sin(a[0]), c2 = cos(a[1]), s2 = sin(a[1]), c3 = cos(a[2]), s3 = sin(a[2]);
  // Rz(a3) * Rx(a2) * Rz(a1), written out; column-major output
  const double r[3][3] = {{c3 * c1 - s3 * c2 * s1, -c3 * s1 - s3 * c2 * c1, s3 * s2},
                          {s3 * c1 + c3 * c2 * s1, -s3 * s1 + c3 * c2 * c1, -c3 * s2},
                          {s2 * s1, s2 * c1, c2}};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) R[i + 3 * j] = r[i][j];
  return EMC_OK;
}

// eulerSearch (coordinates/eulerSearch.m:38-177) walked as BH_alignRaw3d_v2.m:1119-1170.
emc_status emc_euler_search(const char* symmetry, double theta_max, double theta_step, double psi_max,
                            double psi_step, double* out, int* count) {
  if (!symmetry || !count) {
    emc::set_error("emc_euler_search: null argument");
    return EMC_E_ARG;
  }
  bool bipolar = false;
  if (theta_max < 0) {
    theta_max = fabs(theta_max);
    bipolar = true;
  }
  double psi_max_w = 2.0 * psi_max;  // eulerSearch.m:58
  double phi_max = 360.0;
  const char k = symmetry[0];
  const char* num = symmetry + 1;
  // SetSymmetryLimits (eulerSearch.m:126-177)
  if (k == 'C') {
    const double n = atof(num);
    if (!(n >= 1)) { emc::set_error("cyclic symmetry needs C<n>"); return EMC_E_ARG; }
    psi_max_w = fmin(psi_max_w, 360.0 / n);
    theta_max = fmin(180.0, theta_max);
    phi_max = 360.0;
  } else if (k == 'D') {
    const double n = atof(num);
    if (!(n >= 1)) { emc::set_error("dihedral symmetry needs D<n>"); return EMC_E_ARG; }
    psi_max_w = 360.0 / n;
    theta_max = fmin(theta_max, 90.0);
    phi_max = 360.0;
  } else if (k == 'O') {
    if (num[0]) { emc::set_error("octahedral symmetry takes no integer"); return EMC_E_ARG; }
    psi_max_w = fmin(psi_max_w, 90.0);
    theta_max = fmin(theta_max, 54.7);
    phi_max = 90.0;
  } else if (k == 'I') {
    if (num[0] && strcmp(num, "2") != 0) { emc::set_error("icosahedral symmetry is I or I2"); return EMC_E_ARG; }
    psi_max_w = fmin(psi_max_w, 180.0);
    theta_max = 31.7;
    phi_max = 180.0;
  } else {
    emc::set_error("symmetry symbol %s not recognised", symmetry);
    return EMC_E_ARG;
  }
  // CalculateGridSearchPositions (eulerSearch.m:69-124)
  std::vector<double> psi = emc::colon(-psi_max_w / 2.0, psi_step, psi_max_w / 2.0);
  std::vector<double> theta = emc::colon(0.0, theta_step, theta_max);
  if (theta.empty()) theta.push_back(0.0);
  if (bipolar) {
    const size_t n = theta.size();
    for (size_t i = 0; i < n; ++i) theta.push_back(180.0 - theta[n - 1 - i]);
  }
  if (psi.empty()) psi.push_back(0.0);
  int total = 0;
  for (double th : theta) {
    double phi_step;
    if (th == 0.0 || th == 180.0) {
      phi_step = phi_max;
    } else {
      phi_step = fabs(theta_step / sin(th * M_PI / 180.0));
      if (phi_step > phi_max)
        phi_step = phi_max;
      else
        phi_step = phi_max / floor(phi_max / phi_step + 0.5);
    }
    std::vector<double> phi = emc::colon(0.0, phi_step, phi_max - 1.0);
    for (double ph : phi)
      for (double ps : psi) {
        if (out) {
          out[3 * total + 0] = fmod(ph, 360.0);
          out[3 * total + 1] = th;
          out[3 * total + 2] = ps;
        }
        ++total;
      }
  }
  *count = total;
  return EMC_OK;
}

// The symmetry operators the interpolator applies (testScripts/interpolator.m:172-214, used by
// interp3d over iSym = 1:nSymMats):  C<n>: defineMatrix([0, 0, k 360/n], 'Bah', 'forward'),
// k = 0..n-1.  D<n>: the same n in-plane rotations -- check_symmetry also stores their mirrored
// copies (element-wise times [1 -1 1; 1 -1 1; 1 1 -1]) after them, but sets nSymMats = n before
// adding them, so the interpolator never applies the copies.  O: the 24 rotations of the cube
// (the signed permutation matrices of determinant +1, identity first).
emc_status emc_symmetry_matrices(const char* symmetry, double* out, int* count) {
  if (!symmetry || !count) {
    emc::set_error("emc_symmetry_matrices: null argument");
    return EMC_E_ARG;
  }
  std::vector<double> mats;
  const char kind = symmetry[0];
  if (kind == 'C' || kind == 'D') {
    char* end = nullptr;
    const long n = strtol(symmetry + 1, &end, 10);
    if (end == symmetry + 1 || *end != '\0' || n < 1 || n > 30) {
      emc::set_error("emc_symmetry_matrices: '%s' needs an order 1..30", symmetry);
      return EMC_E_ARG;
    }
    const double inc = 360.0 / (double)n;
    for (long k = 0; k < n; ++k) {
      double R[9];
      const double ang[3] = {0.0, 0.0, (double)k * inc};
      const emc_status rs = emc_define_matrix(ang, 0, R);
      if (rs != EMC_OK) return rs;
      mats.insert(mats.end(), R, R + 9);
    }
  } else if (kind == 'O' && symmetry[1] == '\0') {
    const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    const int perm_sign[6] = {1, -1, -1, 1, 1, -1};
    for (int p = 0; p < 6; ++p)
      for (int s = 0; s < 8; ++s) {
        const int sg[3] = {(s & 1) ? -1 : 1, (s & 2) ? -1 : 1, (s & 4) ? -1 : 1};
        if (perm_sign[p] * sg[0] * sg[1] * sg[2] != 1) continue;
        double R[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int i = 0; i < 3; ++i) R[i + 3 * perms[p][i]] = sg[i];  // row i has its entry in column perm[i]
        mats.insert(mats.end(), R, R + 9);
      }
  } else {
    emc::set_error("emc_symmetry_matrices: symmetry '%s' not supported (C<n>, D<n>, O)", symmetry);
    return EMC_E_UNSUPPORTED;
  }
  const int n = (int)(mats.size() / 9);
  if (out) std::copy(mats.begin(), mats.end(), out);
  *count = n;
  return EMC_OK;
}

}  // extern "C"
