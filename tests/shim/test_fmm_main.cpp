// Runs the reference's test/test_fmm.h through the C++ driver shim: test_fmm(p)
// is the potential error of the FMM against direct summation on 10 sampled
// bodies (the 3d/fmm.cxx sequence, N = 10,000, ncrit = 64, theta = 0.4).  The
// reference's GoogleTest wrapper (test/test_fmm.cxx:5-6) asserts < 1e-3 at
// P = 10 and < 1e-6 at P = 20; GoogleTest is not needed for that.
#include "test_fmm.h"

int main() {
  const double e10 = test_fmm(10), e20 = test_fmm(20);
  printf("test_fmm %.9e %.9e\n", e10, e20);
  return e10 < 1e-3 && e20 < 1e-6 ? 0 : 1;
}
