// ljrule.hpp -- Lennard-Jones combination rules, shared by host set-up and
// the device kernels.
#pragma once

namespace qb {

#if defined(__CUDACC__)
#define QB_HD __host__ __device__
#else
#define QB_HD
#endif

// Lennard-Jones coefficients of an atom pair, V = A/r^12 - B/r^6, from the
// two atoms' parameters (a, b) for the pair's LJ code.  Geometric rule
// (nonbond_*): a = sqrt(A_i), b = sqrt(B_i), A = a_i a_j, B = b_i b_j.
// Arithmetic rule (nonbon2_*, md.f90:8972-9089): a = R*_i, b = sqrt(eps_i)
// (square-rooted at set-up), A = b_i b_j (a_i + a_j)^12, B = 2 b_i b_j
// (a_i + a_j)^6, in the reference's order of operations.
QB_HD inline void lj_pair(int arith, double ai, double aj, double bi, double bj, double &A, double &B) {
  if (!arith) {
    A = ai * aj;
    B = bi * bj;
    return;
  }
  double s = ai + aj;
  s = s * s;
  s = s * s * s;
  const double e = bi * bj;
  A = e * s * s;
  B = 2.0 * e * s;
}

}  // namespace qb
