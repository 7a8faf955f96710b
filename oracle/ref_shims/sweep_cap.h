/* Sweep cap of the reference's finetune loops in the capped timing build (oracle/build_reference.py):
 * SBP_REF_MAX_SWEEPS, default 100 (the reference's MAX_NUM_ITERATIONS). */
#pragma once
#include <cstdlib>

inline int sbp_ref_sweep_cap() {
    const char *p = std::getenv("SBP_REF_MAX_SWEEPS");
    const int n = p ? std::atoi(p) : 100;
    return n > 0 ? n : 100;
}
