// TEST INFRASTRUCTURE ONLY: a C ABI over the reference's log-domain path
// score and initial/final choice, compiled from the reference's own header
// (native/string/source_code/legacy_policy.h, included from the reference
// tree by oracle/Makefile `ref`); tests/ compare vext_tst_log_score with it.
#include "legacy_policy.h"

extern "C" int ref_legacy_log_score(const double *a, const double *b, const double *c,
                                    const double *energy, int n, const double *A,
                                    const double *B, const double *C, double T, double mass,
                                    double hop, double *logd) {
    const LegacyLogScore s = legacy_log_score(a, b, c, energy, n, A, B, C, T, mass, hop);
    *logd = s.logd;
    return s.valid ? 1 : 0;
}

extern "C" int ref_legacy_choose_initial(int valid_i, double logd_i, int valid_f,
                                         double logd_f) {
    const LegacyLogScore i = {valid_i != 0, logd_i}, f = {valid_f != 0, logd_f};
    return legacy_choose_initial(i, f) ? 1 : 0;
}
