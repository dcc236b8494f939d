/*
 * LAPACK entry points the reference library references (dense LU/Cholesky/
 * eigen paths, never reached by the sparse solve path) resolved onto SciPy's
 * bundled OpenBLAS, whose exports carry a `scipy_` prefix.  Each symbol is a
 * tail jump, so the argument list passes through unchanged.
 * Test infrastructure only (see oracle/Makefile).
 */
#define FORWARD(name)                                   \
  __asm__(".globl " #name "\n"                          \
          ".type " #name ",@function\n" #name ":\n"     \
          "  jmp scipy_" #name "@PLT\n")
FORWARD(dgetrf_);
FORWARD(dgetrs_);
FORWARD(dsyevd_);
FORWARD(dsygvd_);
FORWARD(dsytrf_);
FORWARD(dsytrs_);
FORWARD(sgetrf_);
FORWARD(sgetrs_);
FORWARD(ssyevd_);
FORWARD(ssygvd_);
FORWARD(ssytrf_);
FORWARD(ssytrs_);
