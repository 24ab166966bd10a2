// Persistent multi-instance kernels (bldm_persist.cuh): float storage, 4-element
// lane vectors, digamma psi_appr; one instantiation per lane shape of
// at most two chunks per lane.
#include "bldm_persist.cuh"

namespace bldm {

#define BLDM_PERSIST_CASE(L, M)                                                           \
    case L * 16 + M:                                                                     \
        return mr ? reinterpret_cast<void*>(&persist_kernel<float, 4, L, M, true, true>)    \
                  : reinterpret_cast<void*>(&persist_kernel<float, 4, L, M, true, false>);

void* pick_persist_f32_v4(int lpf, int mch, bool mr) {
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
