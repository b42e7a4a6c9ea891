// nfft_lean_slice.cuh -- instantiates one slice of the specialized pass
// kernels (NFFT_LEAN_SLICE of NFFT_LEAN_SLICES) so the build compiles the
// slices in parallel.  Each slice registers its kernels with the dispatcher.
#pragma once

#include "nfft_engine.h"
#include "nfft_lean.cuh"
#include "nfft_lean_list.h"

namespace nfft {

template <bool ON, int LOGR, int LOGT, int CI, int CO, int LD, int ST>
struct LeanReg {
    static void add(LeanRegistry&) {}
};
template <int LOGR, int LOGT, int CI, int CO, int LD, int ST>
struct LeanReg<true, LOGR, LOGT, CI, CO, LD, ST> {
    static void add(LeanRegistry& r) {
        r.add(lean_key(LOGR, LOGT, CI, CO, LD, ST),
              (const void*)lean_pass_kernel<real_t, LOGR, LOGT, CI != 0, CO != 0, LD, ST>,
              lean_smem_bytes<real_t, LOGR, LOGT, CI != 0, CO != 0, LD, ST>(), 1 << LOGT);
    }
};

#define NFFT_CAT2(a, b) a##b
#define NFFT_CAT(a, b) NFFT_CAT2(a, b)
#define X(R, T, CI, CO, LD, ST) \
    LeanReg<(__COUNTER__ % NFFT_LEAN_SLICES) == NFFT_LEAN_SLICE, R, T, CI, CO, LD, ST>::add(reg);

void NFFT_CAT(lean_register_slice_, NFFT_LEAN_SLICE)(LeanRegistry& reg) { NFFT_LEAN_ALL(X) }
#undef X

}  // namespace nfft
