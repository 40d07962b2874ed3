// One kernel variant, selected at compile time: PE_MIXED (0 FP64 / 1 mixed / 2 compensated mixed), PE_TPL (threads per Gray lane)
// and PE_KPM (largest cofactor tier the chain kernel contains).  The build compiles this file once
// per variant, in parallel, and links the objects into one library.
#include "fock_kernels.cuh"
#include "fock_registry.h"
#include "fock_warp.cuh"

#if !defined(PE_MIXED) || !defined(PE_TPL) || !defined(PE_KPM)
#error "PE_MIXED, PE_TPL and PE_KPM must be defined"
#endif

namespace {
struct Registration {
    Registration() {
        pe::register_variant(PE_MIXED, PE_TPL, PE_KPM,
                             (void*)pe::fock_chain_kernel<PE_TPL, PE_KPM, PE_MIXED>,
                             (void*)pe::cofactor_kernel<PE_TPL, PE_KPM, PE_MIXED>,
                             (void*)pe::split_partial_kernel<PE_TPL, PE_KPM, PE_MIXED>,
                             (void*)pe::split_draw_kernel<PE_TPL, PE_KPM, PE_MIXED>,
#if PE_KPM <= 16 && PE_TPL <= 2 && PE_MIXED <= 1
                             (void*)pe::fock_chain_warp_kernel<PE_TPL, PE_KPM, (PE_MIXED != 0)>,
                             sizeof(pe::WarpSmemT<PE_KPM>)
#else
                             nullptr, 0
#endif
        );
    }
};
Registration registration;
}  // namespace
