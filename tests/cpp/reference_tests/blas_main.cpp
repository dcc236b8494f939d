// Runs the reference's vector BLAS tests (test/vector/blas/{copy,axpy,xpay,
// axpyz,dot,nrm2}.hpp, used unchanged) against this library's C++ layer,
// at the reference's tolerances (1e-8 double, 1e-4 float).  The tests that
// send their vectors to the device run; the reference's host-only forms
// (vectors never sent) are not applicable here: this library has no CPU
// path and rejects host-resident operands.
#include "axpy.hpp"
#include "axpyz.hpp"
#include "copy.hpp"
#include "dot.hpp"
#include "nrm2.hpp"
#include "xpay.hpp"

#include <cstdlib>

int main(int argc, char **argv) {
  if (argc != 2) {
    std::cout << "usage: " << argv[0] << " size" << std::endl;
    return 1;
  }
  const size_t size = (size_t)std::atol(argv[1]);
  std::cout << "size: " << size << std::endl;
  bool ok = true;
  ok = ok && test_send_copy<double>(size, 1.0e-8) && test_send_copy<float>(size, 1.0e-4);
  ok = ok && test_send_axpy<double>(size, 1.0e-8) && test_send_axpy<float>(size, 1.0e-4);
  ok = ok && test_send_xpay<double>(size, 1.0e-8) && test_send_xpay<float>(size, 1.0e-4);
  ok = ok && test_send_axpyz<double>(size, 1.0e-8) && test_send_axpyz<float>(size, 1.0e-4);
  ok = ok && test_dot<double>(size, 1.0e-8) && test_dot<float>(size, 1.0e-4);
  ok = ok && test_send_dot<double>(size, 1.0e-8) && test_send_dot<float>(size, 1.0e-4);
  ok = ok && test_send_nrm2<double>(size, 1.0e-8) && test_send_nrm2<float>(size, 1.0e-4);
  std::cout << (ok ? "PASS" : "FAIL") << std::endl;
  return ok ? 0 : 1;
}
