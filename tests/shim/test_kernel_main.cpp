// Runs the reference's test/test_kernel.h through the C++ driver shim:
// test_kernel(p) is the potential error of the operator chain P2M -> M2M ->
// M2L -> L2L -> L2P against P2P for one unit charge (single-operator calls).
// The reference's GoogleTest wrapper (test/test_kernel.cxx:5-7) asserts
// < 1e-3, < 1e-6, < 1e-9 at P = 10, 20, 30; GoogleTest is not needed for that.
#include "test_kernel.h"

int main() {
  const double e10 = test_kernel(10), e20 = test_kernel(20), e30 = test_kernel(30);
  printf("test_kernel %.9e %.9e %.9e\n", e10, e20, e30);
  return e10 < 1e-3 && e20 < 1e-6 && e30 < 1e-9 ? 0 : 1;
}
