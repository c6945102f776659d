// ref_adjoint.cpp -- klft's HMC Lie-algebra maps, compiled unchanged from the
// reference tree (-I<reference>/include) on the project's Kokkos-API shim in
// ref_shim/.  TEST INFRASTRUCTURE ONLY: tests/ use it to pin the oracle's
// adjoint projection and exponential map (oracle.cpp adj / expmap) to klft's
// own code, since klft's HMC driver as a whole does not compile.
//
//   AdjointSU2(const SU2 &)   AdjointGroup.hpp:13-19   Adj(M) = (2 Im M01, 2 Re M01, 2 Im M00)
//   exp(const AdjointSU2 &)   AdjointGroup.hpp:98-105  cos|a| + i sin|a| a.sigma / |a|
//   AdjointU1(const U1 &)     AdjointGroup.hpp:114-117 Im M
//   exp(const AdjointU1 &)    AdjointGroup.hpp:170-173 e^{i a}
//   operator*(T, Adjoint*)    AdjointGroup.hpp:92-95, :164-167 (the dtau * P of the gauge update)
//   SU2 / U1 products         GaugeGroup.hpp:376-383, :501-506 (exp(dtau P) * U)
//
// Matrices cross the boundary as interleaved (re, im) doubles in row-major
// order: SU(2) 8 doubles, U(1) 2.
#include <Kokkos_Core.hpp>

#include "AdjointGroup.hpp"

using namespace klft;
using cplx = Kokkos::complex<double>;

namespace {
SU2<double> su2_in(const double *m) {
  return SU2<double>(cplx(m[0], m[1]), cplx(m[2], m[3]), cplx(m[4], m[5]), cplx(m[6], m[7]));
}
void su2_out(const SU2<double> &u, double *m) {
  for (int k = 0; k < 4; ++k) {
    m[2 * k] = u.v[k].real();
    m[2 * k + 1] = u.v[k].imag();
  }
}
}  // namespace

extern "C" {

int ref_su2_adjoint(const double *M, double *v) {
  const AdjointSU2<double> a(su2_in(M));
  for (int k = 0; k < 3; ++k) v[k] = a.v[k];
  return 0;
}

// exp(t * a) as the reference's gauge update forms it
int ref_su2_exp(const double *a, double t, double *U) {
  const AdjointSU2<double> p(a[0], a[1], a[2]);
  su2_out(exp(t * p), U);
  return 0;
}

int ref_su2_mul(const double *A, const double *B, double *C) {
  su2_out(su2_in(A) * su2_in(B), C);
  return 0;
}

int ref_u1_adjoint(const double *M, double *v) {
  const AdjointU1<double> a(U1<double>(cplx(M[0], M[1])));
  v[0] = a.v;
  return 0;
}

int ref_u1_exp(double a, double t, double *U) {
  const AdjointU1<double> p(a);
  const U1<double> u = exp(t * p);
  U[0] = u.v.real();
  U[1] = u.v.imag();
  return 0;
}

}  // extern "C"
