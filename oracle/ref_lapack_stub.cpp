// Link-time stand-in for ProtoMol's Lapack wrapper namespace, used only when
// building the reference as the test oracle.  The wrapper's own non-LAPACK
// fallback (base/Lapack.cpp:48 and following) does not compile as modern
// C++, and nothing on the nonbonded path calls LAPACK; every entry here
// reports that LAPACK is absent.  Signatures follow base/Lapack.h:5-33.
#include <protomol/base/Lapack.h>
#include <stdexcept>

namespace ProtoMol {
namespace Lapack {
static void absent(const char *what) {
  throw std::runtime_error(std::string("LAPACK not built: ") + what);
}
bool isEnabled() { return false; }
void dgemv(char *, int *, int *, double *, double *, int *, double *, int *,
           double *, double *, int *) { absent("dgemv"); }
void dsyev(char *, char *, int *, double *, int *, double *, double *, int *,
           int *) { absent("dsyev"); }
void dsyevr(char *, char *, char *, int *, double *, int *, double *, double *,
            int *, int *, double *, int *, double *, double *, int *, int *,
            double *, int *, int *, int *, int *) { absent("dsyevr"); }
double dlamch(char *) { absent("dlamch"); return 0; }
void dgemm(char *, char *, int *, int *, int *, double *, double *, int *,
           double *, int *, double *, double *, int *) { absent("dgemm"); }
double ddot(int *, double *, int *, double *, int *) { absent("ddot"); return 0; }
double dnrm2(int *, double *, int *) { absent("dnrm2"); return 0; }
void dpotri(char *, int *, double *, int *, int *) { absent("dpotri"); }
void dpotrf(char *, int *, double *, int *, int *) { absent("dpotrf"); }
void dposv(char *, int *, int *, double *, int *, double *, int *, int *) {
  absent("dposv");
}
void dtrmm(char *, char *, char *, char *, int *, int *, double *, double *,
           int *, double *, int *) { absent("dtrmm"); }
void dtrsm(char *, char *, char *, char *, int *, int *, double *, double *,
           int *, double *, int *) { absent("dtrsm"); }
}  // namespace Lapack
}  // namespace ProtoMol
