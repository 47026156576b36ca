// Host-side interfaces shared by the C ABI translation units (hmc_capi.cu, hmc_gsd.cu).
#pragma once

#include <cstdint>

#include "../../include/hmc.h"

namespace hmc {

// Sets the calling thread's hmc_last_error_message() and returns st.
hmc_status report_error(hmc_status st, const char* message);

// One frame of a system's state in FP32 (GSD layout), in pinned host memory owned by the
// system; valid until the next call on the system.
struct GsdFrameView {
    uint64_t step;
    int dim;
    double L[3];
    uint64_t n;
    const float* position;     // n x 3
    const float* orientation;  // n x 4, or null for shapes without orientation
};
hmc_status system_gsd_frame(hmc_system* sys, GsdFrameView* out);

}  // namespace hmc
