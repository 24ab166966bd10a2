// Persistent multi-instance kernels (bldm_persist.cuh): double storage, 2-element
// lane vectors, digamma exact (grad_plus); one instantiation per lane shape of
// at most two chunks per lane.
#include "bldm_persist.cuh"

namespace bldm {

#define BLDM_PERSIST_CASE(L, M)                                                           \
    case L * 16 + M:                                                                     \
        return mr ? reinterpret_cast<void*>(&persist_kernel<double, 2, L, M, false, true>)    \
                  : reinterpret_cast<void*>(&persist_kernel<double, 2, L, M, false, false>);

void* pick_persist_f64_v2_exact(int lpf, int mch, bool mr) {
    switch (lpf * 16 + mch) {
        BLDM_PERSIST_CASE(1, 1)
        BLDM_PERSIST_CASE(2, 1)
        BLDM_PERSIST_CASE(4, 1)
        BLDM_PERSIST_CASE(8, 1)
        BLDM_PERSIST_CASE(16, 1)
        BLDM_PERSIST_CASE(32, 1)
        BLDM_PERSIST_CASE(32, 2)
        default:  // longer fibers (4 or 8 chunks per lane) keep the launch-per-round form
            return nullptr;
    }
}

}  // namespace bldm
