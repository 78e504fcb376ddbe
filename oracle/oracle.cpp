// CPU oracle shared library (the restatement) — TEST INFRASTRUCTURE ONLY.
#define ZORACLE_PREFIX oracle_
#include "oracle_api.H"

ZORACLE_DEFINE_API(zoracle::OracleKernels)

extern "C" void oracle_init_solution(int ncomp, int nx, int ny, const double* lo, const double* hi,
                                     double* v) {
    zoracle::init_solution(ncomp, nx, ny, lo, hi, v);
}
