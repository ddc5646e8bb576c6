// The benchmark problem generator (fvmpor_b200/csrc/problem_gen.cpp, the
// seeded meshes and Ks fields that define the workloads) compiled into the
// oracle's own library, so that a process timing the CPU oracle generates
// its inputs without loading the product library.  Test infrastructure, like
// the rest of oracle/.  The library is linked with -Bsymbolic, so these
// fvm_problem_* symbols bind inside it even when the product library is
// loaded in the same process.
#include "../fvmpor_b200/csrc/problem_gen.cpp"

#include <string>

namespace fvmb {
static thread_local std::string g_orc_problem_error;
void set_error(const std::string& msg) { g_orc_problem_error = msg; }
} // namespace fvmb

extern "C" const char* orc_problem_error(void) { return fvmb::g_orc_problem_error.c_str(); }
